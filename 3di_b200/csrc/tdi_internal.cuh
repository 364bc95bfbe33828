// Internal definitions shared by the kernels and the host driver of the 3DI fitting path.
//
// Arithmetic contract (identical to the CPU oracle): elementwise formulas are evaluated in
// FP32 in the operand order of the 3DI sources with no FMA contraction (this library is
// compiled with -fmad=false; fused multiply-adds appear only where written as fmaf);
// basis x coefficient products are a sequential fused multiply-add over k from 0; sums
// over fragments and landmarks accumulate in FP64; sin/cos/log are evaluated in FP64 and
// rounded to FP32; the Cholesky solve is FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tdi {

constexpr int NL = 51;            // landmarks (src/lib/constants.h:31)
constexpr int DIM = 256;          // crop side (src/lib/constants.h:55-56)
constexpr int NPIX = DIM * DIM;
constexpr int NTMP = 4;           // fragments kept per triangle (src/lib/constants.h:19)
constexpr int KRAD = 7;           // blur radius (src/CMakeLists.txt:1)
constexpr int NTAPS = 2 * KRAD + 1;
constexpr int NMAX = 32768;       // fragment capacity per frame (reference domain: 25,600)
constexpr int TRI_BITS = 20;      // z-buffer key: [13-bit epoch tag | 31-bit depth | 20-bit triangle]
constexpr int TAG_BITS = 64 - 31 - TRI_BITS;
constexpr uint32_t TAG_MAX = (1u << TAG_BITS) - 1;

// words of a per-frame bit set over the triangles
__host__ __device__ constexpr inline int mask_words(int T) { return (T + 31) / 32; }

// frame status bits (same values as the oracle and include/tdi.h)
constexpr uint32_t FLAG_RENDER_SKIPPED = 1u;
constexpr uint32_t FLAG_OUT_OF_DOMAIN = 2u;
constexpr uint32_t FLAG_NAN_DIRECTION = 4u;
constexpr uint32_t FLAG_STUCK_NEG_TZ = 8u;
constexpr uint32_t FLAG_CHOL_FAILED = 16u;
constexpr uint32_t FLAG_FAIL = 32u;
constexpr uint32_t FLAG_OVERFLOW = 64u;       // more fragments than NMAX
constexpr uint32_t FLAG_BAD_INDEX = 128u;     // a triangle corner outside the vertex arrays (skipped)

enum Stage : int32_t { ST_LAMBDA = 0, ST_RIGID = 1, ST_FINETUNE = 2 };
enum Mode : int32_t { M_IDLE = 0, M_FULL = 1, M_TRIAL = 2 };

// Per-frame control block of the batched Gauss-Newton state machine.
struct FrameCtl {
    int32_t active;      // running the current stage
    int32_t mode;        // M_FULL: evaluate at x; M_TRIAL: evaluate at x_ls
    int32_t render;      // render the evaluation point this round
    int32_t need_jac;    // accepted this round: build H, g and a new direction
    float t;             // line-search step
    float obj0;          // objective at x
    float l2base;        // d . g
    int32_t outer;       // num_outer_iters of the running shape fit
    int32_t inner;
    uint32_t flags;
    int32_t N;           // fragments of the last render
    int32_t renders;
    int32_t iters_rigid, iters_finetune, iters_lambda;
    float obj_b;         // barrier objective of the evaluation point (FP32)
    int32_t face_ok;
    uint32_t epoch;      // z-buffer epoch
    double corr;         // correlation sum of the last render
    int32_t bbox[4];     // fragment pixel box of the last raster: xmin, xmax, ymin, ymax
    float objective;     // last accepted objective
    int32_t stage_ok;    // result of the last shape fit (outer > NITERS_SUCCESS)
    int32_t shade_cached;// the light fit's per-fragment shading terms (shc, sht) hold this raster's
};

struct Fragment {        // one surviving fragment, in slot order
    uint32_t pix_owner;  // pixel index (x*256 + y) | owner bit 31
    int32_t tri;
    float al, be;
};

struct Cfg {
    int32_t max_iters_rigid, max_iters_finetune, twostage_illum, finetune, niters_success,
        max_iters_lambda;
    float ref_face_size;
    float taps[NTAPS];
    int32_t normal_eq;       // 0: FP64 in the oracle's order; 1: split-BF16 tensor cores
    float damping;           // lambda of the damped shape solve (H + lambda I), 0 = undamped
    int32_t host_rounds;     // 1: host-driven rounds instead of replayed graphs
    int32_t vertex_stage;    // 0: FP32 fused multiply-add chains; 1: split-BF16 tensor cores
};

// Device view of the model.
// Vertices are numbered internally by slot (Morton order of the mean shape's x-y position);
// tl and lis hold slots. Triangles keep the caller's numbering.
struct DModel {
    int32_t V, T, K, KP;     // KP: K rounded up to a multiple of 4 (row pitch of E)
    int32_t KT, KTP;         // K + 6 unknowns, and its pitch (multiple of 4)
    const float *mean;       // [3][V]
    const float *E;          // [V][3][KP]
    const float *tex;        // [V]
    const int32_t *tl;       // [3][T] corner slots
    const int32_t *lis;      // [NL] landmark slots
    const float *eps_b;      // [4][K]: lb, ub, lb_ft, ub_ft
    const int32_t *tri_order;// [T] triangles in Morton order of their mean-shape centroids
    const int32_t *tlo;      // [3][T] corner slots of the triangles in tri_order
    const int4 *tl4;         // [T] corner slots (b, c, a, 0): one 16-byte gather per triangle
    const int4 *tlo4;        // [T] in tri_order: corner slots and the triangle id (b, c, a, tri)
    const void *Etc;         // the basis split into BF16 pieces in the tensor-core vertex stage's
                             // tile layout (null when K is above that stage's limit)
};

// Device view of a batch of frames and its working set.
struct DBatch {
    int32_t F;               // frames in this batch
    // inputs
    const float *target;     // [F][NPIX] blurred crops
    const float *xl, *yl;    // [F][NL]
    const float *bounds;     // [F][4][NL]
    const float *face_size;  // [F]
    const float *cam;        // [F][4]
    const int32_t *x0y0;     // [F][2]
    const float *Lint;       // [F]
    // state
    float *x, *x_ls, *xe;    // [F][KTP]: accepted, line-search, evaluation point
    float *lam, *lam_ls, *lame, *dlam, *glam;   // [F][4]
    float *d, *g;            // [F][KTP]
    float *H;                // [F][KTP][KTP]
    float *R, *dR;           // [F][9], [F][27] of the evaluation point
    FrameCtl *ctl;           // [F]
    int32_t *act;            // [F] frames running the stage at the start of the round, ascending
    int32_t nact;            // entries of act (host-driven rounds)
    const int32_t *dnact;    // when set: entries of act read from device memory (rounds in a CUDA graph)
    int32_t *rlist;          // [F] frames of act that render this round (after the pre-checks)
    int32_t *rcount;         // [F]: rcount[0] = entries of rlist (one counter per view)
    // per-render working set
    float4 *geo;             // [F][V]: X0, Y0, Z0 and the albedo of the vertex (slot order)
    float4 *proj;            // [F][V]: xp, yp, camera Z, 0 -- what the raster gathers
    unsigned long long *zbuf;// [F][NPIX]
    uint32_t *tri_mask;      // [F][ceil(T/32)] triangles with fragments in the raster in flight
    int32_t *tri_list;       // [F][T] triangles with fragments, ascending
    Fragment *frag;          // [F][NMAX]
    float *fgrad;            // [F][5][NMAX]: gx, gy, h, gxs_n, gys_n
    int32_t *nb;             // [F][4][NMAX]: kl, kr, ka, kb
    float4 *shc;             // [F][NMAX]: unit normal and n . p of each fragment (light fit)
    float *sht;              // [F][NMAX]: interpolated albedo of each fragment (light fit)
    float *J;                // [F][NMAX][KTP]
    double *ne_part;         // [F][NMAX/256][part stride] chunk partials of the normal equations
    float *img;              // [F][2][NPIX] blur scratch for frames too large for shared memory
    // live profiling: frames processed by the kernel being timed (kernel ids as in tdi.h)
    unsigned long long *prof_frames;
    int32_t prof_id;
    int32_t *err;            // [1] nonzero after a device-side wait gave up
};

}  // namespace tdi
