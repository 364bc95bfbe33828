// C ABI and host driver of the batched 3DI fitting path (include/tdi.h).
//
// One batch fits F frames together. Each fitting stage (light fit, shape fit, finetune) is
// a loop of rounds; in a round every frame still running the stage evaluates one point --
// the start of a Gauss-Newton iteration or a line-search trial -- and a per-frame state
// machine on the device applies the reference's decision rules. A frame whose trial is
// accepted gets its normal equations in the same round: the accepted trial's render is the
// render the next outer iteration of the reference would redo at the same point.
#include "tdi_kernels.cu"
#include "tdi_normal_tc.cu"
#include "tdi_vertex_tc.cu"
#include "tdi_preprocess.cu"
#include "tdi_orthographic.cu"
#include "tdi_landmark.cu"
#include "tdi_adjoint.cu"

#include "../../include/tdi.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace tdi;

namespace {

thread_local std::string g_err;

tdi_status fail(tdi_status s, const std::string &msg)
{
    g_err = msg;
    return s;
}

#define TDI_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(TDI_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define TDI_LAUNCH()                                                                       \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess)                                                             \
            return fail(TDI_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_));   \
    } while (0)

inline int round4(int v) { return (v + 3) & ~3; }

// Blur of full crops (the target, video_fitter.cu:548-549): rows then columns, the
// oracle's summation order.
__global__ void k_blur_rows_full(const float *src, float *dst, Cfg c, int F)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)F * NPIX) return;
    const size_t f = i / NPIX;
    const int p = (int)(i - f * NPIX), x = p >> 8, y = p & 255;
    const float *s = src + f * NPIX;
    float acc = 0.0f;
    for (int j = -KRAD; j <= KRAD; ++j) {
        const int yy = y + j;
        const float v = (yy >= 0 && yy < DIM) ? s[x * DIM + yy] : 0.0f;
        acc = acc + c.taps[KRAD - j] * v;
    }
    dst[i] = acc;
}

__global__ void k_blur_cols_full(const float *src, float *dst, Cfg c, int F)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)F * NPIX) return;
    const size_t f = i / NPIX;
    const int p = (int)(i - f * NPIX), x = p >> 8, y = p & 255;
    const float *s = src + f * NPIX;
    float acc = 0.0f;
    for (int j = -KRAD; j <= KRAD; ++j) {
        const int xx = x + j;
        const float v = (xx >= 0 && xx < DIM) ? s[xx * DIM + y] : 0.0f;
        acc = acc + c.taps[KRAD - j] * v;
    }
    dst[i] = acc;
}

__global__ void k_set_render(DBatch b, int frame)
{
    for (int f = threadIdx.x; f < b.F; f += blockDim.x) b.ctl[f].render = (f == frame);
}

__global__ void k_scalars(DBatch b, double *out)   // [F][4]
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.F) return;
    const FrameCtl &c = b.ctl[f];
    out[f * 4 + 0] = c.corr;
    out[f * 4 + 1] = (double)c.obj_b;
    out[f * 4 + 2] = (double)c.obj0;
    out[f * 4 + 3] = (double)c.face_ok;
}

// Configuration values the library cannot run with.
tdi_status check_cfg(const tdi_fit_config &c, const DModel &m)
{
    if (c.normal_eq != 0 && c.normal_eq != 1) return fail(TDI_ERR_INVALID, "normal_eq must be 0 or 1");
    if (!(c.damping >= 0.0f) || !(c.damping < 3.0e38f)) return fail(TDI_ERR_INVALID, "damping must be finite and >= 0");
    if (c.normal_eq == 1 && m.KT + 1 > TC_MAXN)
        return fail(TDI_ERR_INVALID, "tensor-core normal equations take at most 121 expression components");
    if (c.normal_eq == 0 && m.KT + 1 > NE_P8)
        return fail(TDI_ERR_INVALID, "exact normal equations take at most 81 expression components");
    if (c.vertex_stage != 0 && c.vertex_stage != 1) return fail(TDI_ERR_INVALID, "vertex_stage must be 0 or 1");
    if (c.vertex_stage == 1 && !m.Etc)
        return fail(TDI_ERR_INVALID, "the tensor-core vertex stage takes at most 80 expression components");
    return TDI_OK;
}

Cfg to_cfg(const tdi_fit_config &c)
{
    Cfg r;
    r.max_iters_rigid = c.max_iters_rigid;
    r.max_iters_finetune = c.max_iters_finetune;
    r.twostage_illum = c.twostage_illum;
    r.finetune = c.finetune;
    r.niters_success = c.niters_success;
    r.max_iters_lambda = c.max_iters_lambda;
    r.ref_face_size = c.ref_face_size;
    for (int i = 0; i < NTAPS; ++i) r.taps[i] = c.taps[i];
    r.normal_eq = c.normal_eq;
    r.damping = c.damping;
    r.host_rounds = c.host_rounds;
    r.vertex_stage = c.vertex_stage;
    return r;
}

}  // namespace

struct tdi_model {
    DModel d{};
    std::vector<int32_t> vslot;    // internal slot of each vertex
    std::vector<void *> allocs;
    int device = 0;
};

// A lane is a contiguous range of a batch's frames with its own stream and active-frame count:
// the fit runs its lanes' round loops side by side, so that the kernels of one lane fill the
// SMs that the other lane's per-frame kernels leave idle.
struct tdi_lane {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    int *d_count = nullptr;        // [2]: active frames, error word
    int *h_count = nullptr;        // pinned copy
    DBatch d{};                    // view of the lane's frames
    int n = 0;                     // frames running the current stage
};

struct tdi_batch {
    tdi_model *m = nullptr;
    int cap = 0;
    DBatch d{};
    std::vector<tdi_lane> lanes;
    size_t ne_frame_doubles = 0;   // per-frame extent of d.ne_part
    std::vector<void *> allocs;
    float *target_raw = nullptr;   // [cap][NPIX] unblurred upload
    uint8_t *raw_stage = nullptr;  // device copies of raw video frames (tdi_batch_set_video_frames)
    size_t raw_stage_bytes = 0;
    PrepFrame *prep = nullptr;     // [cap] their descriptors
    float *lm_buf = nullptr;       // landmark initialisation: p0L [3][51], orthographic x [cap][7], R [cap][9], slack [cap]
    int32_t *lm_ibuf = nullptr;    // its iterations, run flags, successes, Newton steps [4][cap]
    double *adj = nullptr;         // differentiable loss: FP64 geometry, images, adjoints (tdi_batch_loss)
    size_t adj_doubles = 0;
    float *ctrl_scratch = nullptr;
    double *scalars = nullptr;     // [cap][4]
    int *d_count = nullptr;
    int *h_count = nullptr;        // pinned
    int device = 0;
    int64_t launches = 0;          // kernels launched by this batch
    int prof_id = 0;               // kernel timed by tdi_batch_profile
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
    // CUDA graphs of GRAPH_ROUNDS rounds of a stage, per (lane, stage, capacity tier, frames,
    // config)
    struct RoundGraph {
        int lane, stage, tier, F;
        const FrameCtl *ctl;       // the lane's first frame (its view of the batch)
        Cfg cfg;
        cudaGraphExec_t exec;
        int64_t kernels;           // kernel nodes in the graph
    };
    std::vector<RoundGraph> graphs;
};

namespace {

// Streams a batched fit runs on: lanes are parts of the batch with their own stream, active
// list and round graphs, replayed side by side so that one lane's latency-bound rounds (few
// frames still running, one block per frame) overlap the other's work.
#ifndef TDI_FIT_LANES
#define TDI_FIT_LANES 1
#endif
constexpr int FIT_LANES = TDI_FIT_LANES;
static_assert(FIT_LANES >= 1 && FIT_LANES <= 8, "lanes of a fit");
constexpr int FIT_LANE_MIN = 32;   // frames a lane needs before a batch is split

template <typename T>
tdi_status dalloc(std::vector<void *> &list, T **p, size_t n)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
    if (e != cudaSuccess) return fail(TDI_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    list.push_back(q);
    *p = static_cast<T *>(q);
    return TDI_OK;
}

#define TDI_TRY(x)                        \
    do {                                  \
        tdi_status s_ = (x);              \
        if (s_ != TDI_OK) return s_;      \
    } while (0)

// Launches a kernel of this batch: counts it and, when it is the kernel being profiled,
// brackets it with CUDA events on its stream.
template <typename... KArgs, typename... Args>
tdi_status launch(tdi_batch *bt, int kid, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                  cudaStream_t s, Args... args)
{
    const bool prof = kid != 0 && bt->prof_id == kid;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (prof) {
        TDI_CUDA(cudaEventCreate(&e0));
        TDI_CUDA(cudaEventCreate(&e1));
        TDI_CUDA(cudaEventRecord(e0, s));
    }
    kern<<<grid, block, smem, s>>>(args...);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(TDI_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    bt->launches++;
    if (prof) {
        TDI_CUDA(cudaEventRecord(e1, s));
        bt->prof_events.emplace_back(e0, e1);
    }
    return TDI_OK;
}

// Crop origin from rescaled landmarks (renderer.cu:580-598, padding on).
void crop_origin(const float *xl, const float *yl, int32_t *x0, int32_t *y0)
{
    float xmin = xl[0], xmax = xl[0], ymin = yl[0], ymax = yl[0];
    for (int i = 1; i < NL; ++i) {
        xmin = xl[i] < xmin ? xl[i] : xmin; xmax = xl[i] > xmax ? xl[i] : xmax;
        ymin = yl[i] < ymin ? yl[i] : ymin; ymax = yl[i] > ymax ? yl[i] : ymax;
    }
    const float xs = xmax - xmin, ys = ymax - ymin;
    const float sz = xs > ys ? xs : ys;
    const float fx = (float)((double)xmin - (double)sz / 1.5);
    const float fy = (float)((double)ymin - (double)sz / 1.5);
    *x0 = (int32_t)(uint16_t)(fx > 0.0f ? fx : 0.0f);
    *y0 = (int32_t)(uint16_t)(fy > 0.0f ? fy : 0.0f);
}

float face_size_of(const float *xl, const float *yl)
{
    float xmin = xl[0], xmax = xl[0], ymin = yl[0], ymax = yl[0];
    for (int i = 1; i < NL; ++i) {
        xmin = xl[i] < xmin ? xl[i] : xmin; xmax = xl[i] > xmax ? xl[i] : xmax;
        ymin = yl[i] < ymin ? yl[i] : ymin; ymax = yl[i] > ymax ? yl[i] : ymax;
    }
    const float xs = xmax - xmin, ys = ymax - ymin;
    return xs > ys ? xs : ys;
}


constexpr int ADJ_VERTEX_SMEM_MAX = 100 * 1024;   // the tiled FP64 vertex stage of the loss (K up to ~190)

tdi_status set_attrs()
{
    static bool done = false;
    if (done) return TDI_OK;
    TDI_CUDA(cudaFuncSetAttribute(k_render, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  RENDER_SMEM_FLOATS * (int)sizeof(float)));
    TDI_CUDA(cudaFuncSetAttribute(k_neighbours, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)neigh_smem()));
    TDI_CUDA(cudaFuncSetAttribute(k_vertex_t<VT_FPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TDI_CUDA(cudaFuncSetAttribute(k_vertex_t<VT_FPT_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TDI_CUDA(cudaFuncSetAttribute(k_barrier_full, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TDI_CUDA(cudaFuncSetAttribute(k_solve_t<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TDI_CUDA(cudaFuncSetAttribute(k_solve_t<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TDI_CUDA(cudaFuncSetAttribute(k_normal_eq, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TDI_CUDA(cudaFuncSetAttribute(k_precheck, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TDI_CUDA(cudaFuncSetAttribute(k_normal_eq_tc<NE_GRP>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    TDI_CUDA(cudaFuncSetAttribute(k_normal_eq_tc<TC_MAXN / 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    TDI_CUDA(cudaFuncSetAttribute(k_vertex_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vc_smem(VC_MAXK)));
    TDI_CUDA(cudaFuncSetAttribute(k_adj_vertex_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, ADJ_VERTEX_SMEM_MAX));
    done = true;
    return TDI_OK;
}

// Vertex stage grid: frame tiles of nf frames x vertex-tile groups, about VT_BLOCKS_PER_SM
// blocks per SM.
dim3 vertex_grid(const DModel &m, int frames, int nf = VT_F)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    // the kernel splits the blocks between frame tiles and vertex stripes by the number of
    // frames that render, which is at most `frames`
    const long ftiles = std::max(1, (frames + nf - 1) / nf);
    const long ntiles = (m.V + VT_V - 1) / VT_V;
    return dim3((unsigned)std::max(ftiles, std::min((long)VT_BLOCKS_PER_SM * sms, ftiles * ntiles)));
}

// The exact vertex stage for at most `frames` rendering frames: 8 frames per thread (64-frame
// tiles) for full rounds; 2 per thread (16-frame tiles) when at most VT_SMALL frames can render,
// where a 64-frame tile would carry mostly idle frames through every multiply-add.
constexpr int VT_SMALL = 32;

template <class B>
tdi_status launch_vertex(B *bt, const DModel &m, const DBatch &d, cudaStream_t s, int frames)
{
    if (frames <= VT_SMALL)
        return launch(bt, KID_VERTEX, k_vertex_t<VT_FPT_SMALL>, vertex_grid(m, frames, 8 * VT_FPT_SMALL),
                      dim3(32, VT_WARPS + 1), vt_smem(m.KP, 8 * VT_FPT_SMALL), s, m, d);
    return launch(bt, KID_VERTEX, k_vertex_t<VT_FPT>, vertex_grid(m, frames), dim3(32, VT_WARPS + 1),
                  vt_smem(m.KP), s, m, d);
}

// Tensor-core vertex stage: one block per SM, split between frame tiles and vertex stripes.
dim3 vertex_tc_grid(const DModel &m, int frames)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    const long ftiles = std::max(1, (frames + VC_F - 1) / VC_F);
    const long ntiles = (m.V + VC_V - 1) / VC_V;
    return dim3((unsigned)std::max(ftiles, std::min((long)sms, ftiles * ntiles)));
}

// Blocks per frame of the depth pass: 16, or more when few frames run, so that a short
// launch still spreads over every SM (about five resident blocks per SM).
unsigned raster_blocks(int frames)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    const int want = (5 * sms + std::max(frames, 1) - 1) / std::max(frames, 1);
    return (unsigned)std::max(RD_BLOCKS, std::min(RD_MAX_BLOCKS, want));
}

struct Launch {
    tdi_batch *bt;
    const DModel &m;
    const DBatch &b;
    cudaStream_t s;
    int F;
    size_t smem_neigh() const { return neigh_smem(); }
    size_t smem_ne() const { return (size_t)2 * 2 * NE_SUB * NE_PD * sizeof(double); }
    size_t smem_bar() const { return (size_t)4 * NL * NE_P8 * sizeof(float); }
    size_t smem_solve() const { return solve_smem(m.KT); }
    dim3 fblocks() const { return dim3((F + 127) / 128); }
    int A() const { return b.nact; }                      // frames active this round
    dim3 ablocks() const { return dim3((A() + 127) / 128); }
    dim3 wblocks() const { return dim3((A() + 3) / 4); }      // a warp per active frame, 128 threads
};

// View of frames [f0, f0 + nf) of a batch: every per-frame array starts at frame f0.
DBatch batch_view(const tdi_batch *bt, int f0, int nf)
{
    const DModel &m = bt->m->d;
    const DBatch &a = bt->d;
    const size_t F0 = (size_t)f0, KTP = m.KTP;
    DBatch v = a;
    v.F = nf;
    v.target = a.target + F0 * NPIX;
    v.xl = a.xl + F0 * NL; v.yl = a.yl + F0 * NL;
    v.bounds = a.bounds + F0 * 4 * NL;
    v.face_size = a.face_size + F0;
    v.cam = a.cam + F0 * 4;
    v.x0y0 = a.x0y0 + F0 * 2;
    v.Lint = a.Lint + F0;
    v.x = a.x + F0 * KTP; v.x_ls = a.x_ls + F0 * KTP; v.xe = a.xe + F0 * KTP;
    v.lam = a.lam + F0 * 4; v.lam_ls = a.lam_ls + F0 * 4; v.lame = a.lame + F0 * 4;
    v.dlam = a.dlam + F0 * 4; v.glam = a.glam + F0 * 4;
    v.d = a.d + F0 * KTP; v.g = a.g + F0 * KTP;
    v.H = a.H + F0 * KTP * KTP;
    v.R = a.R + F0 * 9; v.dR = a.dR + F0 * 27;
    v.ctl = a.ctl + F0;
    v.act = a.act + F0;
    v.nact = 0;
    v.rlist = a.rlist + F0;
    v.rcount = a.rcount + F0;
    v.geo = a.geo + F0 * m.V; v.proj = a.proj + F0 * m.V;
    v.zbuf = a.zbuf + F0 * NPIX;
    v.tri_mask = a.tri_mask + F0 * mask_words(m.T);
    v.tri_list = a.tri_list + F0 * m.T;
    v.frag = a.frag + F0 * NMAX;
    v.fgrad = a.fgrad + F0 * 5 * NMAX;
    v.nb = a.nb + F0 * 4 * NMAX;
    v.shc = a.shc + F0 * NMAX; v.sht = a.sht + F0 * NMAX;
    v.J = a.J + F0 * NMAX * KTP;
    v.ne_part = a.ne_part + F0 * bt->ne_frame_doubles;
    v.img = a.img + F0 * RIMG;
    return v;
}

// Compacts a lane's list of frames running the stage; the count arrives with the lane's
// next synchronisation (one 8-byte read-back per round and lane).
tdi_status lane_compact(tdi_batch *bt, tdi_lane &ln)
{
    TDI_TRY(launch(bt, 0, k_compact_active, dim3(1), dim3(1024), 0, ln.s, (const DBatch)ln.d, ln.d_count));
    TDI_CUDA(cudaMemcpyAsync(ln.h_count, ln.d_count, 2 * sizeof(int), cudaMemcpyDeviceToHost, ln.s));
    return TDI_OK;
}

tdi_status lane_count(tdi_lane &ln)
{
    TDI_CUDA(cudaStreamSynchronize(ln.s));
    if (ln.h_count[1]) return fail(TDI_ERR_CUDA, "a bounded device-side wait gave up (error word set)");
    ln.n = ln.h_count[0];
    ln.d.nact = ln.n;
    return TDI_OK;
}

// Compacts the list of frames running the stage and returns how many there are (one 4-byte
// read-back per call).
tdi_status compact_active(tdi_batch *bt, cudaStream_t s, int *n)
{
    TDI_TRY(launch(bt, 0, k_compact_active, dim3(1), dim3(1024), 0, s, (const DBatch)bt->d, bt->d_count));
    TDI_CUDA(cudaMemcpyAsync(bt->h_count, bt->d_count, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    TDI_CUDA(cudaStreamSynchronize(s));
    if (bt->h_count[1]) return fail(TDI_ERR_CUDA, "a bounded device-side wait gave up (error word set)");
    *n = *bt->h_count;
    bt->d.nact = *n;
    return TDI_OK;
}

tdi_status geometry(const Launch &L, const Cfg &c, int stage)
{
    // the pre-render checks need only the landmarks: a rejected trial skips the vertex stage
    TDI_TRY(launch(L.bt, 0, k_precheck, dim3((L.A() + PC_WARPS - 1) / PC_WARPS), dim3(PC_WARPS * 32),
                   precheck_smem(L.m.K, L.m.KP), L.s, L.m, L.b, c, stage));
    TDI_TRY(launch(L.bt, 0, k_compact_render, dim3(1), dim3(1024), 0, L.s, L.b));
    if (c.vertex_stage == 1)
        TDI_TRY(launch(L.bt, KID_VERTEX, k_vertex_tc, vertex_tc_grid(L.m, L.A()), dim3(VC_THREADS), vc_smem(L.m.K),
                       L.s, L.m, L.b, reinterpret_cast<const __nv_bfloat16 *>(L.m.Etc)));
    else
        TDI_TRY(launch_vertex(L.bt, L.m, L.b, L.s, L.A()));
    TDI_TRY(launch(L.bt, KID_RASTER, k_raster_depth, dim3(raster_blocks(L.A()), L.A()), dim3(RD_THREADS), 0, L.s, L.m, L.b));
    TDI_TRY(launch(L.bt, KID_RESOLVE, k_raster_resolve, dim3(L.A()), dim3(RR_THREADS), 0, L.s, L.m, L.b));
    return TDI_OK;
}

tdi_status render(const Launch &L, const Cfg &c, int stage)
{
    return launch(L.bt, KID_RENDER, k_render, dim3(L.A()), dim3(RENDER_THREADS),
                  RENDER_SMEM_FLOATS * sizeof(float), L.s, L.m, L.b, c, stage);
}

tdi_status normal_equations(const Launch &L, const Cfg &c, int stage)
{
    TDI_TRY(launch(L.bt, KID_NEIGHBOURS, k_neighbours, dim3(L.A()), dim3(1024), L.smem_neigh(), L.s, L.b, 0));
    TDI_TRY(launch(L.bt, KID_JACOBIAN, k_jacobian, dim3(JAC_BPF, L.A()), dim3(JAC_THREADS), 0, L.s, L.m, L.b));
    if (c.normal_eq == 1) {
        // column groups of 8 per thread: 11 cover the reference's 79 expressions and the
        // weight column
        if (L.m.KT + 1 <= 8 * NE_GRP)
            TDI_TRY(launch(L.bt, KID_NORMAL_EQ, k_normal_eq_tc<NE_GRP>, dim3(TC_BPF, L.A()), dim3(TC_THREADS),
                           (size_t)TC_SMEM, L.s, L.m, L.b));
        else
            TDI_TRY(launch(L.bt, KID_NORMAL_EQ, k_normal_eq_tc<TC_MAXN / 8>, dim3(TC_BPF, L.A()), dim3(TC_THREADS),
                           (size_t)TC_SMEM, L.s, L.m, L.b));
        TDI_TRY(launch(L.bt, 0, k_normal_eq_tc_reduce, dim3(TC_RBLOCKS, L.A()), dim3(256), 0, L.s, L.m, L.b));
    } else {
        TDI_TRY(launch(L.bt, KID_NORMAL_EQ, k_normal_eq, dim3(NE_BPF, L.A()), dim3(NE_THREADS), L.smem_ne(), L.s, L.m, L.b));
        TDI_TRY(launch(L.bt, 0, k_normal_eq_reduce, dim3(4, L.A()), dim3(NE_THREADS), 0, L.s, L.m, L.b));
    }
    TDI_TRY(launch(L.bt, KID_BARRIER, k_barrier_full, dim3(L.A()), dim3(256), L.smem_bar(), L.s, L.m, L.b,
                   (int)(stage == ST_FINETUNE)));
    TDI_TRY(launch(L.bt, KID_SOLVE, L.m.KT <= 96 ? k_solve_t<6> : k_solve_t<8>, dim3(L.A()), dim3(SV_THREADS),
                   L.smem_solve(), L.s, L.m, L.b, c, stage));
    return TDI_OK;
}

// One round of a stage for the frames of b (launched on s).
tdi_status stage_round(tdi_batch *bt, const Cfg &c, int stage, const DBatch &b, cudaStream_t s, long round)
{
    const DModel &m = bt->m->d;
    Launch L{bt, m, b, s, b.F};
    TDI_TRY(launch(bt, 0, k_prepare, L.wblocks(), dim3(128), 0, s, m, b, stage));
    if (stage == ST_LAMBDA) {
        if (round == 0) {
            TDI_TRY(geometry(L, c, stage));
            TDI_TRY(launch(bt, KID_NEIGHBOURS, k_neighbours, dim3(L.A()), dim3(1024), L.smem_neigh(), s, b, 1));
        }
        TDI_TRY(render(L, c, stage));
        TDI_TRY(launch(bt, 0, k_decide_lambda, L.ablocks(), dim3(128), 0, s, m, b, c));
        TDI_TRY(launch(bt, 0, k_lambda_jac, dim3(L.A()), dim3(256), 0, s, m, b, c));
    } else {
        TDI_TRY(geometry(L, c, stage));
        TDI_TRY(render(L, c, stage));
        TDI_TRY(launch(bt, 0, k_decide_shape, L.ablocks(), dim3(128), 0, s, m, b, c, stage));
        TDI_TRY(normal_equations(L, c, stage));
    }
    return TDI_OK;
}

// Rounds replayed from CUDA graphs. A graph holds GRAPH_ROUNDS rounds of a stage, each followed by
// the compaction of the active frames into the device count that the next round's kernels
// read; grids are sized for a capacity tier (the smallest of 32, 128, 512 or the batch that
// holds the frames still running: the count only falls during a stage), and blocks past the
// device count return at once. The host reads the count once per replay instead of once per
// round. Graphs are built on first use and kept per (stage, tier, frames, configuration).
constexpr int GRAPH_ROUNDS = 16;

int graph_tier(int n, int F)
{
    for (int t : {32, 128, 512})
        if (n <= t && t < F) return t;
    return F;
}

tdi_status stage_graph(tdi_batch *bt, const Cfg &c, int stage, int lane, int tier, tdi_batch::RoundGraph **out)
{
    tdi_lane &ln = bt->lanes[lane];
    for (auto &g : bt->graphs)
        if (g.lane == lane && g.stage == stage && g.tier == tier && g.F == ln.d.F && g.ctl == ln.d.ctl &&
            std::memcmp(&g.cfg, &c, sizeof(Cfg)) == 0) {
            *out = &g;
            return TDI_OK;
        }
    DBatch gv = ln.d;
    gv.dnact = ln.d_count;
    gv.nact = tier;                             // grid sizes only: the kernels read the device count
    const int64_t before = bt->launches;
    TDI_CUDA(cudaStreamBeginCapture(ln.s, cudaStreamCaptureModeThreadLocal));
    tdi_status st = TDI_OK;
    for (int r = 0; r < GRAPH_ROUNDS && st == TDI_OK; ++r) {
        st = stage_round(bt, c, stage, gv, ln.s, 1 + r);
        if (st == TDI_OK)
            st = launch(bt, 0, k_compact_active, dim3(1), dim3(1024), 0, ln.s, (const DBatch)gv, ln.d_count);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(ln.s, &graph);
    const int64_t kernels = bt->launches - before;
    bt->launches = before;
    if (st != TDI_OK) { if (graph) cudaGraphDestroy(graph); return st; }
    if (ec != cudaSuccess) return fail(TDI_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(TDI_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    bt->graphs.push_back({lane, stage, tier, ln.d.F, ln.d.ctl, c, exec, kernels});
    *out = &bt->graphs.back();
    return TDI_OK;
}

// A stage with its rounds replayed from graphs (no live profiling): every lane's replay is
// enqueued on its stream before any lane's count is read back.
tdi_status run_stage_graphs(tdi_batch *bt, const Cfg &c, int stage, int nlanes)
{
    const DModel &m = bt->m->d;
    for (int l = 0; l < nlanes; ++l) {
        tdi_lane &ln = bt->lanes[l];
        TDI_TRY(launch(bt, 0, k_stage_start, dim3((ln.d.F + 127) / 128), dim3(128), 0, ln.s, m, ln.d, c, stage));
        TDI_TRY(lane_compact(bt, ln));
    }
    for (int l = 0; l < nlanes; ++l) TDI_TRY(lane_count(bt->lanes[l]));
    const long max_rounds = stage == ST_LAMBDA ? 8L * c.max_iters_lambda + 16
                                               : 16L * (stage == ST_RIGID ? c.max_iters_rigid : c.max_iters_finetune) + 16;
    long round[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (stage == ST_LAMBDA) {                   // the light fit's first round also rasterises
        for (int l = 0; l < nlanes; ++l) {
            tdi_lane &ln = bt->lanes[l];
            if (ln.n <= 0) continue;
            TDI_TRY(stage_round(bt, c, stage, ln.d, ln.s, 0));
            TDI_TRY(lane_compact(bt, ln));
            round[l] = 1;
        }
        for (int l = 0; l < nlanes; ++l)
            if (round[l]) TDI_TRY(lane_count(bt->lanes[l]));
    }
    for (;;) {
        bool launched[8] = {false, false, false, false, false, false, false, false}, any = false;
        for (int l = 0; l < nlanes; ++l) {
            tdi_lane &ln = bt->lanes[l];
            if (ln.n <= 0 || round[l] >= max_rounds) continue;
            tdi_batch::RoundGraph *g = nullptr;
            TDI_TRY(stage_graph(bt, c, stage, l, graph_tier(ln.n, ln.d.F), &g));
            TDI_CUDA(cudaGraphLaunch(g->exec, ln.s));
            bt->launches += g->kernels;
            TDI_CUDA(cudaMemcpyAsync(ln.h_count, ln.d_count, 2 * sizeof(int), cudaMemcpyDeviceToHost, ln.s));
            round[l] += GRAPH_ROUNDS;
            launched[l] = any = true;
        }
        if (!any) break;
        for (int l = 0; l < nlanes; ++l)
            if (launched[l]) TDI_TRY(lane_count(bt->lanes[l]));
    }
    return TDI_OK;
}

// A stage (fit_3DMM_lambdas / _shape_rigid / _epsilon_finetune) for every frame of every lane:
// the lanes' rounds are enqueued on their own streams before any lane is waited for.
tdi_status run_stage_lanes(tdi_batch *bt, const Cfg &c, int stage, int nlanes)
{
    if (!c.host_rounds && bt->prof_id == 0) return run_stage_graphs(bt, c, stage, nlanes);
    const DModel &m = bt->m->d;
    for (int l = 0; l < nlanes; ++l) {
        tdi_lane &ln = bt->lanes[l];
        TDI_TRY(launch(bt, 0, k_stage_start, dim3((ln.d.F + 127) / 128), dim3(128), 0, ln.s, m, ln.d, c, stage));
        TDI_TRY(lane_compact(bt, ln));
    }
    for (int l = 0; l < nlanes; ++l) TDI_TRY(lane_count(bt->lanes[l]));
    const long max_rounds = stage == ST_LAMBDA ? 8L * c.max_iters_lambda + 16
                                               : 16L * (stage == ST_RIGID ? c.max_iters_rigid : c.max_iters_finetune) + 16;
    for (long round = 0; round < max_rounds; ++round) {
        bool any = false;
        for (int l = 0; l < nlanes; ++l) {
            tdi_lane &ln = bt->lanes[l];
            if (ln.n <= 0) continue;
            any = true;
            TDI_TRY(stage_round(bt, c, stage, ln.d, ln.s, round));
            TDI_TRY(lane_compact(bt, ln));
        }
        if (!any) break;
        for (int l = 0; l < nlanes; ++l)
            if (bt->lanes[l].n > 0) TDI_TRY(lane_count(bt->lanes[l]));
    }
    return TDI_OK;
}

__global__ void k_fit_begin(DBatch b)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.F) return;
    FrameCtl &c = b.ctl[f];
    c.flags = 0;
    c.iters_rigid = c.iters_finetune = c.iters_lambda = 0;
    c.renders = 0;
    c.stage_ok = 0;
    c.objective = 0.0f;
    c.N = 0;
}

__global__ void k_fit_end(DBatch b)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.F) return;
    FrameCtl &c = b.ctl[f];
    if (!c.stage_ok) c.flags |= FLAG_FAIL;
}

}  // namespace

extern "C" {

const char *tdi_last_error(void) { return g_err.c_str(); }

tdi_status tdi_model_create(const tdi_model_desc *desc, tdi_model **out)
{
    if (!desc || !out) return fail(TDI_ERR_INVALID, "null argument");
    const int V = desc->n_vertices, T = desc->n_triangles, K = desc->n_expr;
    if (V <= 0 || T <= 0 || K <= 0 || K > 500 || !desc->mean || !desc->expr_basis || !desc->tex ||
        !desc->triangles || !desc->landmarks || !desc->eps_lb || !desc->eps_ub ||
        !desc->eps_lb_finetune || !desc->eps_ub_finetune)
        return fail(TDI_ERR_INVALID, "incomplete model description");
    if (T >= (1 << TRI_BITS)) return fail(TDI_ERR_INVALID, "too many triangles");
    for (int i = 0; i < 3 * T; ++i)
        if (desc->triangles[i] < 0 || desc->triangles[i] >= V) return fail(TDI_ERR_INVALID, "triangle index out of range");
    for (int i = 0; i < NL; ++i)
        if (desc->landmarks[i] < 0 || desc->landmarks[i] >= V) return fail(TDI_ERR_INVALID, "landmark index out of range");
    TDI_TRY(set_attrs());
    tdi_model *m = new tdi_model();
    cudaGetDevice(&m->device);
    DModel &d = m->d;
    d.V = V; d.T = T; d.K = K; d.KP = round4(K); d.KT = K + 6; d.KTP = round4(K + 6);
    float *mean, *E, *tex, *epsb;
    int32_t *tl, *lis, *order, *tlo;
    int4 *tl4, *tlo4;
    auto cleanup = [&](tdi_status st) { for (void *p : m->allocs) cudaFree(p); delete m; return st; };
    tdi_status st;
    if ((st = dalloc(m->allocs, &mean, 3 * (size_t)V)) || (st = dalloc(m->allocs, &E, (size_t)V * 3 * d.KP)) ||
        (st = dalloc(m->allocs, &tex, (size_t)V)) || (st = dalloc(m->allocs, &tl, 3 * (size_t)T)) ||
        (st = dalloc(m->allocs, &lis, (size_t)NL)) || (st = dalloc(m->allocs, &epsb, 4 * (size_t)K)) ||
        (st = dalloc(m->allocs, &order, (size_t)T)) || (st = dalloc(m->allocs, &tlo, 3 * (size_t)T)) ||
        (st = dalloc(m->allocs, &tl4, (size_t)T)) || (st = dalloc(m->allocs, &tlo4, (size_t)T)))
        return cleanup(st);
    // Internal vertex numbering: vertices are stored in Morton order of their mean-shape (x, y)
    // position (slot), so that the corners of neighbouring triangles sit in neighbouring
    // memory. Every per-vertex quantity is computed independently of the numbering; the
    // entry points that take or return per-vertex arrays translate at the boundary.
    // The raster's depth pass visits triangles in Morton order of their centroids (the
    // z-buffer result does not depend on the order); tlo holds their corners as slots.
    float xmin = desc->mean[0], xmax = xmin, ymin = desc->mean[V], ymax = ymin;
    for (int v = 0; v < V; ++v) {
        xmin = std::min(xmin, desc->mean[v]); xmax = std::max(xmax, desc->mean[v]);
        ymin = std::min(ymin, desc->mean[V + v]); ymax = std::max(ymax, desc->mean[V + v]);
    }
    const float sx = 65535.0f / std::max(xmax - xmin, 1e-20f), sy = 65535.0f / std::max(ymax - ymin, 1e-20f);
    auto spread = [](uint32_t x) {
        x &= 0xFFFF;
        x = (x | (x << 8)) & 0x00FF00FFu; x = (x | (x << 4)) & 0x0F0F0F0Fu;
        x = (x | (x << 2)) & 0x33333333u; x = (x | (x << 1)) & 0x55555555u;
        return x;
    };
    auto morton = [&](float x, float y) {
        const uint32_t qx = (uint32_t)std::min(65535.0f, std::max(0.0f, (x - xmin) * sx));
        const uint32_t qy = (uint32_t)std::min(65535.0f, std::max(0.0f, (y - ymin) * sy));
        return spread(qx) | (spread(qy) << 1);
    };
    m->vslot.resize(V);
    std::vector<int32_t> vord(V);
    {
        std::vector<std::pair<uint32_t, int32_t>> keys(V);
        for (int v = 0; v < V; ++v) keys[v] = {morton(desc->mean[v], desc->mean[V + v]), v};
        std::sort(keys.begin(), keys.end());
        for (int s = 0; s < V; ++s) { vord[s] = keys[s].second; m->vslot[keys[s].second] = s; }
    }
    std::vector<int32_t> tord(T), tls(3 * (size_t)T), tlo_h(3 * (size_t)T), lis_h(NL);
    {
        std::vector<std::pair<uint32_t, int32_t>> keys(T);
        for (int t = 0; t < T; ++t) {
            float cx = 0.0f, cy = 0.0f;
            for (int r = 0; r < 3; ++r) {
                const int v = desc->triangles[r * T + t];
                cx += desc->mean[v]; cy += desc->mean[V + v];
            }
            keys[t] = {morton(cx / 3.0f, cy / 3.0f), t};
        }
        std::sort(keys.begin(), keys.end());
        for (int t = 0; t < T; ++t) tord[t] = keys[t].second;
    }
    for (int r = 0; r < 3; ++r)
        for (int t = 0; t < T; ++t) tls[(size_t)r * T + t] = m->vslot[desc->triangles[(size_t)r * T + t]];
    for (int r = 0; r < 3; ++r)
        for (int s = 0; s < T; ++s) tlo_h[(size_t)r * T + s] = tls[(size_t)r * T + tord[s]];
    for (int i = 0; i < NL; ++i) lis_h[i] = m->vslot[desc->landmarks[i]];
    std::vector<int4> tl4_h(T), tlo4_h(T);
    for (int t = 0; t < T; ++t) tl4_h[t] = make_int4(tls[t], tls[(size_t)T + t], tls[2 * (size_t)T + t], 0);
    for (int s2 = 0; s2 < T; ++s2) tlo4_h[s2] = make_int4(tlo_h[s2], tlo_h[(size_t)T + s2], tlo_h[2 * (size_t)T + s2], tord[s2]);
    std::vector<float> mean_h(3 * (size_t)V), tex_h(V);
    for (int c = 0; c < 3; ++c)
        for (int s = 0; s < V; ++s) mean_h[(size_t)c * V + s] = desc->mean[(size_t)c * V + vord[s]];
    for (int s = 0; s < V; ++s) tex_h[s] = desc->tex[vord[s]];
    std::vector<float> Ep((size_t)V * 3 * d.KP, 0.0f);
    for (int s = 0; s < V; ++s)
        for (int c = 0; c < 3; ++c)
            std::memcpy(&Ep[((size_t)s * 3 + c) * d.KP], desc->expr_basis + ((size_t)vord[s] * 3 + c) * K, sizeof(float) * K);
    std::vector<float> eb(4 * (size_t)K);
    std::memcpy(&eb[0], desc->eps_lb, sizeof(float) * K);
    std::memcpy(&eb[K], desc->eps_ub, sizeof(float) * K);
    std::memcpy(&eb[2 * K], desc->eps_lb_finetune, sizeof(float) * K);
    std::memcpy(&eb[3 * K], desc->eps_ub_finetune, sizeof(float) * K);
    if (cudaMemcpy(mean, mean_h.data(), sizeof(float) * 3 * V, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(E, Ep.data(), sizeof(float) * Ep.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(tex, tex_h.data(), sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(tl, tls.data(), sizeof(int32_t) * 3 * T, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(lis, lis_h.data(), sizeof(int32_t) * NL, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(epsb, eb.data(), sizeof(float) * eb.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(order, tord.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(tlo, tlo_h.data(), sizeof(int32_t) * 3 * T, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(tl4, tl4_h.data(), sizeof(int4) * T, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(tlo4, tlo4_h.data(), sizeof(int4) * T, cudaMemcpyHostToDevice) != cudaSuccess)
        return cleanup(fail(TDI_ERR_CUDA, "model upload failed"));
    d.mean = mean; d.E = E; d.tex = tex; d.tl = tl; d.lis = lis; d.eps_b = epsb; d.tri_order = order; d.tlo = tlo; d.tl4 = tl4; d.tlo4 = tlo4;
    if (K <= VC_MAXK) {
        // the basis split into BF16 pieces once, in the tensor-core vertex stage's tile layout
        const int ntiles = (V + VC_V - 1) / VC_V;
        uint8_t *etc = nullptr;
        if ((st = dalloc(m->allocs, &etc, (size_t)ntiles * vc_tile_bytes(K)))) return cleanup(st);
        k_split_basis<<<1024, 256>>>(d, ntiles, reinterpret_cast<__nv_bfloat16 *>(etc));
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
            return cleanup(fail(TDI_ERR_CUDA, "basis split failed"));
        d.Etc = etc;
    }
    *out = m;
    return TDI_OK;
}

tdi_status tdi_model_destroy(tdi_model *m)
{
    if (!m) return TDI_OK;
    for (void *p : m->allocs) cudaFree(p);
    delete m;
    return TDI_OK;
}

tdi_status tdi_batch_create(tdi_model *m, int32_t max_frames, tdi_batch **out)
{
    if (!m || !out || max_frames <= 0) return fail(TDI_ERR_INVALID, "bad batch arguments");
    tdi_batch *b = new tdi_batch();
    b->m = m;
    b->cap = max_frames;
    cudaGetDevice(&b->device);
    const DModel &md = m->d;
    DBatch &d = b->d;
    const size_t F = (size_t)max_frames, KTP = md.KTP;
    auto cleanup = [&](tdi_status st) {
        for (void *p : b->allocs) cudaFree(p);
        if (b->h_count) cudaFreeHost(b->h_count);
        delete b;
        return st;
    };
    float *target, *xl, *yl, *bounds, *fs, *cam, *Lint;
    int32_t *x0y0;
    tdi_status st = TDI_OK;
#define A(ptr, n) if (st == TDI_OK) st = dalloc(b->allocs, &ptr, (n))
    A(target, F * NPIX); A(b->target_raw, F * NPIX); A(b->prep, F); A(xl, F * NL); A(yl, F * NL);
    A(bounds, F * 4 * NL); A(fs, F); A(cam, F * 4); A(x0y0, F * 2); A(Lint, F);
    A(d.x, F * KTP); A(d.x_ls, F * KTP); A(d.xe, F * KTP);
    A(d.lam, F * 4); A(d.lam_ls, F * 4); A(d.lame, F * 4); A(d.dlam, F * 4); A(d.glam, F * 4);
    A(d.d, F * KTP); A(d.g, F * KTP); A(d.H, F * KTP * KTP); A(d.R, F * 9); A(d.dR, F * 27);
    A(d.ctl, F); A(d.act, F); A(d.rlist, F); A(d.rcount, F); A(d.geo, F * (size_t)md.V); A(d.proj, F * (size_t)md.V); A(d.zbuf, F * NPIX); A(d.tri_mask, F * (size_t)mask_words(md.T)); A(d.tri_list, F * (size_t)md.T); A(d.frag, F * NMAX);
    A(d.fgrad, F * 5 * NMAX); A(d.nb, F * 4 * NMAX); A(d.shc, F * NMAX); A(d.sht, F * NMAX);
    A(d.J, F * NMAX * KTP); b->ne_frame_doubles = NE_MAXCH * std::max((size_t)ne_part_stride((int)KTP), (tc_part_bytes(md.KT) + 7) / 8);
    A(d.ne_part, F * b->ne_frame_doubles); A(d.err, 1); A(d.img, F * RIMG); A(b->scalars, F * 4); A(b->d_count, 2);
    A(d.prof_frames, 1);
#undef A
    if (st != TDI_OK) return cleanup(st);
    if (cudaMallocHost(&b->h_count, 2 * sizeof(int)) != cudaSuccess) return cleanup(fail(TDI_ERR_NOMEM, "pinned alloc"));
    if (cudaMemset(d.zbuf, 0xFF, F * NPIX * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(d.ctl, 0, F * sizeof(FrameCtl)) != cudaSuccess ||
        cudaMemset(d.err, 0, sizeof(int32_t)) != cudaSuccess ||
        cudaMemset(d.tri_mask, 0, F * mask_words(md.T) * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(d.x, 0, F * KTP * sizeof(float)) != cudaSuccess ||
        cudaMemset(d.x_ls, 0, F * KTP * sizeof(float)) != cudaSuccess ||
        cudaMemset(d.J, 0, F * NMAX * KTP * sizeof(float)) != cudaSuccess ||
        cudaMemset(d.prof_frames, 0, sizeof(unsigned long long)) != cudaSuccess)
        return cleanup(fail(TDI_ERR_CUDA, "batch init failed"));
    d.F = max_frames;
    d.target = target; d.xl = xl; d.yl = yl; d.bounds = bounds; d.face_size = fs; d.cam = cam;
    d.x0y0 = x0y0; d.Lint = Lint;
    d.prof_id = 0;
    // lanes: two for batches that can be halved, each with a non-blocking stream
    b->lanes.resize(max_frames >= 2 ? FIT_LANES : 1);
    for (auto &ln : b->lanes) {
        if (cudaStreamCreateWithFlags(&ln.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ln.ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost(&ln.h_count, 2 * sizeof(int)) != cudaSuccess ||
            dalloc(b->allocs, &ln.d_count, 2) != TDI_OK) {
            tdi_batch_destroy(b);
            return fail(TDI_ERR_CUDA, "lane creation failed");
        }
    }
    *out = b;
    return TDI_OK;
}

tdi_status tdi_batch_destroy(tdi_batch *b)
{
    if (!b) return TDI_OK;
    for (auto &g : b->graphs) cudaGraphExecDestroy(g.exec);
    for (auto &e : b->prof_events) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    for (auto &ln : b->lanes) {
        if (ln.s) cudaStreamDestroy(ln.s);
        if (ln.ev) cudaEventDestroy(ln.ev);
        if (ln.h_count) cudaFreeHost(ln.h_count);
    }
    for (void *p : b->allocs) cudaFree(p);
    if (b->raw_stage) cudaFree(b->raw_stage);
    if (b->lm_buf) cudaFree(b->lm_buf);
    if (b->lm_ibuf) cudaFree(b->lm_ibuf);
    if (b->adj) cudaFree(b->adj);
    if (b->h_count) cudaFreeHost(b->h_count);
    delete b;
    return TDI_OK;
}

// Landmarks, bounds, cameras, crop origins and face sizes of a batch's frames (not the crops).
static tdi_status set_frames_meta(tdi_batch *b, const tdi_frames *fr, cudaStream_t s)
{
    const int F = fr->n_frames;
    b->d.F = F;
    std::vector<int32_t> x0y0(2 * (size_t)F);
    std::vector<float> fs(F);
    for (int f = 0; f < F; ++f) {
        if (fr->x0y0) { x0y0[2 * f] = fr->x0y0[2 * f]; x0y0[2 * f + 1] = fr->x0y0[2 * f + 1]; }
        else crop_origin(fr->xl + f * NL, fr->yl + f * NL, &x0y0[2 * f], &x0y0[2 * f + 1]);
        fs[f] = fr->face_size ? fr->face_size[f] : face_size_of(fr->xl + f * NL, fr->yl + f * NL);
    }
    DBatch &d = b->d;
    TDI_CUDA(cudaMemcpyAsync((void *)d.xl, fr->xl, sizeof(float) * NL * F, cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaMemcpyAsync((void *)d.yl, fr->yl, sizeof(float) * NL * F, cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaMemcpyAsync((void *)d.bounds, fr->bounds, sizeof(float) * 4 * NL * F, cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaMemcpyAsync((void *)d.cam, fr->cam, sizeof(float) * 4 * F, cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaMemcpyAsync((void *)d.x0y0, x0y0.data(), sizeof(int32_t) * 2 * F, cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaMemcpyAsync((void *)d.face_size, fs.data(), sizeof(float) * F, cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaStreamSynchronize(s));   // the host vectors above go out of scope
    return TDI_OK;
}

tdi_status tdi_batch_set_frames(tdi_batch *b, const tdi_frames *fr, void *stream)
{
    if (!b || !fr || !fr->targets || !fr->xl || !fr->yl || !fr->bounds || !fr->cam)
        return fail(TDI_ERR_INVALID, "incomplete frames");
    if (fr->n_frames <= 0) return fail(TDI_ERR_INVALID, "no frames");
    if (fr->n_frames > b->cap) return fail(TDI_ERR_CAPACITY, "more frames than the batch holds");
    cudaStream_t s = (cudaStream_t)stream;
    TDI_CUDA(cudaMemcpyAsync(b->target_raw, fr->targets, sizeof(float) * NPIX * fr->n_frames, cudaMemcpyHostToDevice, s));
    return set_frames_meta(b, fr, s);
}

// Raw video frames (video_fitter.cu:520-550, input_data.cu:32-53, camera.h:162-174): each
// frame is rescaled by c = ref_face_size / face_size (float division), landmarks and camera
// by c (float products), the crop origin and face size are taken from the rescaled
// landmarks, and the crop is formed on the device (k_preprocess). Frames are staged on the
// device in groups that fit PP_STAGE_BYTES.
constexpr size_t PP_STAGE_BYTES = (size_t)256 << 20;

tdi_status tdi_batch_set_video_frames(tdi_batch *b, const tdi_video_frames *fr, void *stream)
{
    if (!b || !fr || !fr->bgr || !fr->xp || !fr->yp || !fr->bounds || !fr->face_size || !fr->cam)
        return fail(TDI_ERR_INVALID, "incomplete video frames");
    if (fr->n_frames <= 0) return fail(TDI_ERR_INVALID, "no frames");
    if (fr->n_frames > b->cap) return fail(TDI_ERR_CAPACITY, "more frames than the batch holds");
    if (fr->width <= 0 || fr->height <= 0 || fr->row_bytes < 3 * (int64_t)fr->width)
        return fail(TDI_ERR_INVALID, "bad image size or row pitch");
    if (!fr->ref_face_sizes && !(fr->ref_face_size > 0.0f)) return fail(TDI_ERR_INVALID, "ref_face_size must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    const int F = fr->n_frames;
    std::vector<float> xl((size_t)F * NL), yl((size_t)F * NL), cam((size_t)F * 4);
    std::vector<PrepFrame> pf(F);
    for (int f = 0; f < F; ++f) {
        const float ref = fr->ref_face_sizes ? fr->ref_face_sizes[f] : fr->ref_face_size;
        if (!(fr->face_size[f] > 0.0f) || !(ref > 0.0f)) return fail(TDI_ERR_INVALID, "face sizes must be positive");
        const float c = ref / fr->face_size[f];
        for (int i = 0; i < NL; ++i) {
            xl[(size_t)f * NL + i] = c * fr->xp[(size_t)f * NL + i];
            yl[(size_t)f * NL + i] = c * fr->yp[(size_t)f * NL + i];
        }
        for (int q = 0; q < 4; ++q) cam[(size_t)f * 4 + q] = fr->cam[(size_t)f * 4 + q] * c;
        PrepFrame &p = pf[f];
        p.row_bytes = fr->row_bytes;
        p.width = fr->width;
        p.height = fr->height;
        // cv::resize: dsize = round(size * c) in double, source step 1 / c in double
        p.rw = (int32_t)std::nearbyint((double)fr->width * (double)c);
        p.rh = (int32_t)std::nearbyint((double)fr->height * (double)c);
        p.inv = 1.0 / (double)c;
        crop_origin(&xl[(size_t)f * NL], &yl[(size_t)f * NL], &p.x0, &p.y0);
    }
    tdi_frames tf{};
    tf.n_frames = F;
    tf.targets = nullptr;
    tf.xl = xl.data();
    tf.yl = yl.data();
    tf.bounds = fr->bounds;
    tf.face_size = nullptr;
    tf.cam = cam.data();
    tf.x0y0 = nullptr;
    TDI_TRY(set_frames_meta(b, &tf, s));
    const size_t fbytes = (size_t)fr->height * (size_t)fr->row_bytes;
    const int group = (int)std::max<size_t>(1, std::min<size_t>((size_t)F, PP_STAGE_BYTES / std::max<size_t>(fbytes, 1)));
    if (b->raw_stage_bytes < fbytes * group) {
        TDI_CUDA(cudaStreamSynchronize(s));
        if (b->raw_stage) { cudaFree(b->raw_stage); b->raw_stage = nullptr; b->raw_stage_bytes = 0; }
        TDI_CUDA(cudaMalloc(&b->raw_stage, fbytes * group));
        b->raw_stage_bytes = fbytes * group;
    }
    for (int f0 = 0; f0 < F; f0 += group) {
        const int n = std::min(group, F - f0);
        TDI_CUDA(cudaMemcpyAsync(b->raw_stage, fr->bgr + (size_t)f0 * fbytes, fbytes * n, cudaMemcpyHostToDevice, s));
        for (int f = f0; f < f0 + n; ++f) pf[f].bgr = b->raw_stage + (size_t)(f - f0) * fbytes;
        TDI_CUDA(cudaMemcpyAsync(b->prep + f0, pf.data() + f0, sizeof(PrepFrame) * n, cudaMemcpyHostToDevice, s));
        TDI_TRY(launch(b, 0, k_preprocess, dim3(DIM / PP_TILE, DIM / PP_TILE, n), dim3(PP_TILE, PP_ROWS), 0, s,
                       (const PrepFrame *)(b->prep + f0), b->target_raw + (size_t)f0 * NPIX));
        TDI_CUDA(cudaStreamSynchronize(s));   // the stage is reused by the next group
    }
    return TDI_OK;
}

static tdi_status blur_targets(tdi_batch *b, const Cfg &c, cudaStream_t s)
{
    const size_t n = (size_t)b->d.F * NPIX;
    const dim3 blocks((unsigned)((n + 255) / 256));
    TDI_TRY(launch(b, 0, k_blur_rows_full, blocks, dim3(256), 0, s, (const float *)b->target_raw, b->d.img, c, b->d.F));
    // img holds 2*NPIX floats per frame; the row pass above used the first F*NPIX floats
    TDI_TRY(launch(b, 0, k_blur_cols_full, blocks, dim3(256), 0, s, (const float *)b->d.img, (float *)b->d.target, c, b->d.F));
    return TDI_OK;
}

tdi_status tdi_batch_set_state(tdi_batch *b, const float *x, const float *lam, const float *L, void *stream)
{
    if (!b || !lam || !L) return fail(TDI_ERR_INVALID, "null state");
    cudaStream_t s = (cudaStream_t)stream;
    const DModel &m = b->m->d;
    const int F = b->d.F;
    std::vector<float> xp((size_t)F * m.KTP, 0.0f), lp((size_t)F * 4, 0.0f);
    for (int f = 0; f < F; ++f) {
        if (x) std::memcpy(&xp[(size_t)f * m.KTP], x + (size_t)f * m.KT, sizeof(float) * m.KT);
        for (int j = 0; j < 3; ++j) lp[f * 4 + j] = lam[f * 3 + j];
    }
    if (x) {   // NULL keeps the states on the device (after tdi_batch_landmark_init)
        TDI_CUDA(cudaMemcpyAsync(b->d.x, xp.data(), sizeof(float) * xp.size(), cudaMemcpyHostToDevice, s));
        TDI_CUDA(cudaMemcpyAsync(b->d.x_ls, xp.data(), sizeof(float) * xp.size(), cudaMemcpyHostToDevice, s));
    }
    TDI_CUDA(cudaMemcpyAsync(b->d.lam, lp.data(), sizeof(float) * lp.size(), cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaMemcpyAsync(b->d.lam_ls, lp.data(), sizeof(float) * lp.size(), cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaMemcpyAsync((void *)b->d.Lint, L, sizeof(float) * F, cudaMemcpyHostToDevice, s));
    TDI_CUDA(cudaStreamSynchronize(s));
    return TDI_OK;
}

tdi_status tdi_batch_fit(tdi_batch *b, const tdi_fit_config *cfg, void *stream)
{
    if (!b || !cfg) return fail(TDI_ERR_INVALID, "null argument");
    TDI_TRY(check_cfg(*cfg, b->m->d));
    cudaStream_t s = (cudaStream_t)stream;
    const Cfg c = to_cfg(*cfg);
    const dim3 fb((b->d.F + 127) / 128);
    TDI_TRY(blur_targets(b, c, s));
    TDI_TRY(launch(b, 0, k_fit_begin, fb, dim3(128), 0, s, b->d));
    // lanes: halves of the batch on their own streams, ordered after the work on s
    const int F = b->d.F;
    const int nlanes = std::min((int)b->lanes.size(), F >= 2 * FIT_LANE_MIN ? FIT_LANES : 1);
    TDI_CUDA(cudaEventRecord(b->lanes[0].ev, s));
    for (int l = 0; l < nlanes; ++l) {
        tdi_lane &ln = b->lanes[l];
        const int f0 = (int)((long)F * l / nlanes), f1 = (int)((long)F * (l + 1) / nlanes);
        ln.d = batch_view(b, f0, f1 - f0);
        TDI_CUDA(cudaStreamWaitEvent(ln.s, b->lanes[0].ev, 0));
    }
    TDI_TRY(run_stage_lanes(b, c, ST_LAMBDA, nlanes));
    TDI_TRY(run_stage_lanes(b, c, ST_RIGID, nlanes));
    if (c.twostage_illum) {
        for (int k = 0; k < 2; ++k) {
            TDI_TRY(run_stage_lanes(b, c, ST_LAMBDA, nlanes));
            TDI_TRY(run_stage_lanes(b, c, ST_RIGID, nlanes));
        }
    }
    if (c.finetune) TDI_TRY(run_stage_lanes(b, c, ST_FINETUNE, nlanes));
    for (int l = 0; l < nlanes; ++l) {
        TDI_CUDA(cudaEventRecord(b->lanes[l].ev, b->lanes[l].s));
        TDI_CUDA(cudaStreamWaitEvent(s, b->lanes[l].ev, 0));
    }
    TDI_TRY(launch(b, 0, k_fit_end, fb, dim3(128), 0, s, b->d));
    return TDI_OK;
}

tdi_status tdi_batch_get_state(tdi_batch *b, float *x, float *lam, tdi_report *rep, void *stream)
{
    if (!b) return fail(TDI_ERR_INVALID, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    const DModel &m = b->m->d;
    const int F = b->d.F;
    std::vector<float> xp((size_t)F * m.KTP), lp((size_t)F * 4);
    std::vector<FrameCtl> ctl(F);
    TDI_CUDA(cudaMemcpyAsync(xp.data(), b->d.x, sizeof(float) * xp.size(), cudaMemcpyDeviceToHost, s));
    TDI_CUDA(cudaMemcpyAsync(lp.data(), b->d.lam, sizeof(float) * lp.size(), cudaMemcpyDeviceToHost, s));
    TDI_CUDA(cudaMemcpyAsync(ctl.data(), b->d.ctl, sizeof(FrameCtl) * F, cudaMemcpyDeviceToHost, s));
    TDI_CUDA(cudaStreamSynchronize(s));
    for (int f = 0; f < F; ++f) {
        if (x) std::memcpy(x + (size_t)f * m.KT, &xp[(size_t)f * m.KTP], sizeof(float) * m.KT);
        if (lam) for (int j = 0; j < 3; ++j) lam[f * 3 + j] = lp[f * 4 + j];
        if (rep) {
            rep[f].flags = ctl[f].flags;
            rep[f].n_fragments = ctl[f].N;
            rep[f].iters_rigid = ctl[f].iters_rigid;
            rep[f].iters_finetune = ctl[f].iters_finetune;
            rep[f].iters_lambda = ctl[f].iters_lambda;
            rep[f].renders = ctl[f].renders;
            rep[f].objective = ctl[f].objective;
        }
    }
    return TDI_OK;
}

tdi_status tdi_fit_frames(tdi_batch *b, const tdi_frames *frames, const tdi_fit_config *cfg,
                          float *x, float *lam, const float *L, tdi_report *rep, void *stream)
{
    TDI_TRY(tdi_batch_set_frames(b, frames, stream));
    TDI_TRY(tdi_batch_set_state(b, x, lam, L, stream));
    TDI_TRY(tdi_batch_fit(b, cfg, stream));
    return tdi_batch_get_state(b, x, lam, rep, stream);
}

tdi_status tdi_batch_evaluate(tdi_batch *b, const tdi_fit_config *cfg, int32_t finetune_bounds, void *stream)
{
    if (!b || !cfg) return fail(TDI_ERR_INVALID, "null argument");
    TDI_TRY(check_cfg(*cfg, b->m->d));
    cudaStream_t s = (cudaStream_t)stream;
    const Cfg c = to_cfg(*cfg);
    const DModel &m = b->m->d;
    const DBatch &d = b->d;
    Launch L{b, m, d, s, d.F};
    const int stage = finetune_bounds ? ST_FINETUNE : ST_RIGID;
    TDI_TRY(blur_targets(b, c, s));
    TDI_TRY(launch(b, 0, k_fit_begin, L.fblocks(), dim3(128), 0, s, d));
    TDI_TRY(launch(b, 0, k_stage_start, L.fblocks(), dim3(128), 0, s, m, d, c, stage));
    int n = 0;
    TDI_TRY(compact_active(b, s, &n));
    if (n == 0) return TDI_OK;
    TDI_TRY(launch(b, 0, k_prepare, L.wblocks(), dim3(128), 0, s, m, d, stage));
    TDI_TRY(geometry(L, c, stage));
    TDI_TRY(render(L, c, stage));
    TDI_TRY(launch(b, 0, k_decide_shape, L.ablocks(), dim3(128), 0, s, m, d, c, stage));
    TDI_TRY(normal_equations(L, c, stage));
    TDI_TRY(launch(b, 0, k_scalars, L.fblocks(), dim3(128), 0, s, d, b->scalars));
    TDI_CUDA(cudaStreamSynchronize(s));
    return TDI_OK;
}

// Euler angles in degrees of a column-major rotation (rotation_header.cu:421-449, RAD2DEG of
// constants.h:59): atan2 in double, rounded to float.
static void euler_degrees(const float *R, float *ypr)
{
    const float c = std::sqrt(R[5] * R[5] + R[8] * R[8]);
    float yaw, pitch, roll;
    if (!(c < 1e-6f)) {
        roll = (float)std::atan2((double)R[1], (double)R[0]);
        yaw = (float)std::atan2((double)-R[2], (double)c);
        pitch = (float)std::atan2((double)R[5], (double)R[8]);
    } else {
        roll = (float)std::atan2((double)-R[7], (double)R[4]);
        yaw = (float)std::atan2((double)-R[2], (double)c);
        pitch = 0.0f;
    }
    ypr[0] = (float)((double)(yaw * 180.0f) / M_PI);
    ypr[1] = (float)((double)(pitch * 180.0f) / M_PI);
    ypr[2] = (float)((double)(roll * 180.0f) / M_PI);
}

tdi_status tdi_apply_identity(int32_t n_vertices, int32_t n_id, int32_t n_tex, const float *mean0,
                              const float *id_basis, const float *alpha, const float *tex0,
                              const float *tex_basis, const float *beta, float *mean, float *tex,
                              void *stream)
{
    if (n_vertices <= 0 || n_id < 0 || n_tex < 0 || !mean0 || !tex0 || !mean || !tex ||
        (n_id > 0 && (!id_basis || !alpha)) || (n_tex > 0 && (!tex_basis || !beta)))
        return fail(TDI_ERR_INVALID, "bad identity arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t V = (size_t)n_vertices, KA = (size_t)n_id, KB = (size_t)n_tex;
    const size_t nf = 4 * V + 3 * V * KA + KA + V * KB + KB;
    float *buf = nullptr;
    TDI_CUDA(cudaMalloc(&buf, nf * sizeof(float)));
    float *dm = buf, *dt = dm + 3 * V, *dI = dt + V, *da = dI + 3 * V * KA, *dT = da + KA, *db = dT + V * KB;
    auto run = [&]() -> tdi_status {
        TDI_CUDA(cudaMemcpyAsync(dm, mean0, 3 * V * sizeof(float), cudaMemcpyHostToDevice, s));
        TDI_CUDA(cudaMemcpyAsync(dt, tex0, V * sizeof(float), cudaMemcpyHostToDevice, s));
        if (KA) {
            TDI_CUDA(cudaMemcpyAsync(dI, id_basis, 3 * V * KA * sizeof(float), cudaMemcpyHostToDevice, s));
            TDI_CUDA(cudaMemcpyAsync(da, alpha, KA * sizeof(float), cudaMemcpyHostToDevice, s));
        }
        if (KB) {
            TDI_CUDA(cudaMemcpyAsync(dT, tex_basis, V * KB * sizeof(float), cudaMemcpyHostToDevice, s));
            TDI_CUDA(cudaMemcpyAsync(db, beta, KB * sizeof(float), cudaMemcpyHostToDevice, s));
        }
        const unsigned blocks = (unsigned)((4 * V + 255) / 256);
        k_apply_identity<<<blocks, 256, 0, s>>>((int)V, (int)KA, (int)KB, dm, dI, da, dt, dT, db);
        TDI_CUDA(cudaGetLastError());
        TDI_CUDA(cudaMemcpyAsync(mean, dm, 3 * V * sizeof(float), cudaMemcpyDeviceToHost, s));
        TDI_CUDA(cudaMemcpyAsync(tex, dt, V * sizeof(float), cudaMemcpyDeviceToHost, s));
        TDI_CUDA(cudaStreamSynchronize(s));
        return TDI_OK;
    };
    const tdi_status st = run();
    cudaFree(buf);
    return st;
}

tdi_status tdi_orthographic_init(int32_t n_frames, const float *xl, const float *yl, const float *p0L,
                                 float *x_out, float *ypr_out, int32_t *iters_out, void *stream)
{
    if (n_frames <= 0 || !xl || !yl || !p0L || !x_out) return fail(TDI_ERR_INVALID, "bad orthographic arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t F = (size_t)n_frames;
    const size_t nf = 2 * F * NL + 3 * NL + F * OR_N + F * 9;
    float *dbuf = nullptr;
    int32_t *dit = nullptr;
    TDI_CUDA(cudaMalloc(&dbuf, nf * sizeof(float)));
    if (cudaMalloc(&dit, F * sizeof(int32_t)) != cudaSuccess) { cudaFree(dbuf); return fail(TDI_ERR_CUDA, "cudaMalloc"); }
    float *dxl = dbuf, *dyl = dxl + F * NL, *dp = dyl + F * NL, *dx = dp + 3 * NL, *dR = dx + F * OR_N;
    std::vector<float> R(F * 9);
    std::vector<int32_t> it(F);
    tdi_status st = TDI_OK;
    auto run = [&]() -> tdi_status {
        TDI_CUDA(cudaMemcpyAsync(dxl, xl, F * NL * sizeof(float), cudaMemcpyHostToDevice, s));
        TDI_CUDA(cudaMemcpyAsync(dyl, yl, F * NL * sizeof(float), cudaMemcpyHostToDevice, s));
        TDI_CUDA(cudaMemcpyAsync(dp, p0L, 3 * NL * sizeof(float), cudaMemcpyHostToDevice, s));
        k_orthographic<<<(unsigned)((F + OR_WARPS - 1) / OR_WARPS), OR_WARPS * 32, 0, s>>>(dxl, dyl, dp, n_frames, dx, dR, dit,
                                                                                     nullptr, nullptr);
        TDI_CUDA(cudaGetLastError());
        TDI_CUDA(cudaMemcpyAsync(x_out, dx, F * OR_N * sizeof(float), cudaMemcpyDeviceToHost, s));
        TDI_CUDA(cudaMemcpyAsync(R.data(), dR, F * 9 * sizeof(float), cudaMemcpyDeviceToHost, s));
        TDI_CUDA(cudaMemcpyAsync(it.data(), dit, F * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        TDI_CUDA(cudaStreamSynchronize(s));
        return TDI_OK;
    };
    st = run();
    cudaFree(dbuf);
    cudaFree(dit);
    if (st != TDI_OK) return st;
    for (size_t f = 0; f < F; ++f) {
        if (ypr_out) euler_degrees(&R[f * 9], ypr_out + f * 3);
        if (iters_out) iters_out[f] = it[f];
    }
    return TDI_OK;
}

tdi_status tdi_batch_landmark_init(tdi_batch *b, const float *p0L, int32_t *success, float *slack, int32_t *iters,
                                   void *stream)
{
    if (!b || !p0L) return fail(TDI_ERR_INVALID, "null argument");
    const DModel &m = b->m->d;
    if (m.K + 7 > LM_MAXN) return fail(TDI_ERR_INVALID, "landmark initialisation takes at most 129 expression components");
    const int F = b->d.F;
    if (F <= 0) return fail(TDI_ERR_INVALID, "no frames: call tdi_batch_set_frames first");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t cap = (size_t)b->cap;
    if (!b->lm_buf) {
        TDI_CUDA(cudaMalloc(&b->lm_buf, sizeof(float) * (3 * NL + cap * (7 + 9 + 1))));
        if (cudaMalloc(&b->lm_ibuf, sizeof(int32_t) * 4 * cap) != cudaSuccess) {
            cudaFree(b->lm_buf);
            b->lm_buf = nullptr;
            return fail(TDI_ERR_NOMEM, "cudaMalloc");
        }
    }
    float *dp = b->lm_buf, *xo = dp + 3 * NL, *Ro = xo + 7 * cap, *dslack = Ro + 9 * cap;
    int32_t *dit = b->lm_ibuf, *drun = dit + cap, *dsucc = drun + cap, *dnewton = dsucc + cap;
    static bool attr = false;
    if (!attr) {
        TDI_CUDA(cudaFuncSetAttribute(k_landmark_init, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        attr = true;
    }
    const size_t smem = lm_smem(m.K);
    if (smem > 220 * 1024) return fail(TDI_ERR_INVALID, "too many expression components for the landmark fit");
    TDI_CUDA(cudaMemcpyAsync(dp, p0L, sizeof(float) * 3 * NL, cudaMemcpyHostToDevice, s));
    const unsigned ob = (unsigned)((F + OR_WARPS - 1) / OR_WARPS);
    TDI_TRY(launch(b, 0, k_orthographic, dim3(ob), dim3(OR_WARPS * 32), 0, s, (const float *)b->d.xl,
                   (const float *)b->d.yl, (const float *)dp, F, xo, Ro, dit, (const float *)nullptr,
                   (const int32_t *)nullptr));
    TDI_TRY(launch(b, 0, k_lm_flip, dim3((F + 127) / 128), dim3(128), 0, s, F, xo, (const float *)Ro, drun));
    TDI_TRY(launch(b, 0, k_orthographic, dim3(ob), dim3(OR_WARPS * 32), 0, s, (const float *)b->d.xl,
                   (const float *)b->d.yl, (const float *)dp, F, xo, Ro, dit, (const float *)xo, (const int32_t *)drun));
    TDI_TRY(launch(b, 0, k_landmark_init, dim3(F), dim3(LM_THREADS), smem, s, m, b->d, (const float *)xo, dsucc,
                   dslack, dnewton));
    if (success) TDI_CUDA(cudaMemcpyAsync(success, dsucc, sizeof(int32_t) * F, cudaMemcpyDeviceToHost, s));
    if (slack) TDI_CUDA(cudaMemcpyAsync(slack, dslack, sizeof(float) * F, cudaMemcpyDeviceToHost, s));
    if (iters) TDI_CUDA(cudaMemcpyAsync(iters, dnewton, sizeof(int32_t) * F, cudaMemcpyDeviceToHost, s));
    TDI_CUDA(cudaStreamSynchronize(s));
    if (b->h_count) {
        int32_t e = 0;
        TDI_CUDA(cudaMemcpy(&e, b->d.err, sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (e) return fail(TDI_ERR_CUDA, "a bounded device-side wait gave up (error word set)");
    }
    return TDI_OK;
}

// Working set of the differentiable loss for cap frames, carved from one FP64 allocation.
struct AdjBufs {
    double *geo, *R, *img, *tmp, *B, *T, *adjB, *adjI, *dP0, *dpos, *glob, *geps, *loss;
};

static tdi_status adj_bufs(tdi_batch *b, AdjBufs &o)
{
    const DModel &m = b->m->d;
    const size_t F = (size_t)b->cap, V = (size_t)m.V;
    const size_t sizes[13] = {F * V * 8, F * 36, F * NPIX, F * NPIX, F * NPIX, F * NPIX, F * NPIX, F * NPIX,
                              F * V * 3, F * V * 2, F * AD_GLOB, F * (size_t)m.K, F};
    size_t total = 0;
    for (size_t s : sizes) total += (s + 31) / 32 * 32;
    if (!b->adj) {
        TDI_CUDA(cudaMalloc(&b->adj, total * sizeof(double)));
        b->adj_doubles = total;
    }
    double **dst[13] = {&o.geo, &o.R, &o.img, &o.tmp, &o.B, &o.T, &o.adjB, &o.adjI, &o.dP0, &o.dpos, &o.glob, &o.geps, &o.loss};
    double *p = b->adj;
    for (int i = 0; i < 13; ++i) { *dst[i] = p; p += (sizes[i] + 31) / 32 * 32; }
    return TDI_OK;
}

// The raster at the caller's states and the FP64 loss (the forward of the loss and of its adjoint).
static tdi_status adj_forward(tdi_batch *b, const Cfg &c, const float *x, const float *lam, const float *L,
                              cudaStream_t s, AdjBufs &o)
{
    const DModel &m = b->m->d;
    DBatch &d = b->d;
    const int F = d.F;
    TDI_TRY(adj_bufs(b, o));
    Launch Lc{b, m, d, s, F};
    TDI_TRY(launch(b, 0, k_adj_set_x, dim3((F * m.KT + 255) / 256), dim3(256), 0, s, m, d, x, F));
    TDI_TRY(launch(b, 0, k_fit_begin, Lc.fblocks(), dim3(128), 0, s, d));
    TDI_TRY(launch(b, 0, k_stage_start, Lc.fblocks(), dim3(128), 0, s, m, d, c, (int)ST_RIGID));
    int n = 0;
    TDI_TRY(compact_active(b, s, &n));
    if (n > 0) {
        TDI_TRY(launch(b, 0, k_prepare, Lc.wblocks(), dim3(128), 0, s, m, d, (int)ST_RIGID));
        TDI_TRY(launch(b, 0, k_compact_render, dim3(1), dim3(1024), 0, s, (const DBatch)d));
        TDI_TRY(launch_vertex(b, m, d, s, n));
        TDI_TRY(launch(b, KID_RASTER, k_raster_depth, dim3(raster_blocks(n), n), dim3(RD_THREADS), 0, s, m, d));
        TDI_TRY(launch(b, KID_RESOLVE, k_raster_resolve, dim3(n), dim3(RR_THREADS), 0, s, m, d));
    }
    const size_t np = (size_t)F * NPIX;
    const dim3 pb((unsigned)((np + 255) / 256));
    TDI_TRY(launch(b, 0, k_adj_rot, dim3((F + 127) / 128), dim3(128), 0, s, m, d, x, F, o.R));
    if (adj_vertex_smem(m.KP) <= (size_t)ADJ_VERTEX_SMEM_MAX)
        TDI_TRY(launch(b, 0, k_adj_vertex_tiled, dim3((m.V + AV_V - 1) / AV_V, (F + AV_F - 1) / AV_F), dim3(256),
                       adj_vertex_smem(m.KP), s, m, x, F, (const double *)o.R, (const float *)d.cam, o.geo));
    else
        TDI_TRY(launch(b, 0, k_adj_vertex, dim3((m.V + 255) / 256, F), dim3(256), 0, s, m, x, F, (const double *)o.R,
                       (const float *)d.cam, o.geo));
    TDI_CUDA(cudaMemsetAsync(o.img, 0, np * sizeof(double), s));
    TDI_TRY(launch(b, 0, k_adj_shade, dim3(16, F), dim3(AD_THREADS), 0, s, m, (const DBatch)d, x, lam, L, F,
                   (const double *)o.geo, (const double *)o.R, o.img));
    TDI_TRY(launch(b, 0, k_adj_blur, pb, dim3(256), 0, s, (const double *)o.img, o.tmp, c, F, 0));
    TDI_TRY(launch(b, 0, k_adj_blur, pb, dim3(256), 0, s, (const double *)o.tmp, o.B, c, F, 1));
    TDI_TRY(launch(b, 0, k_adj_widen, pb, dim3(256), 0, s, (const float *)b->target_raw, o.img, np));
    TDI_TRY(launch(b, 0, k_adj_blur, pb, dim3(256), 0, s, (const double *)o.img, o.tmp, c, F, 0));
    TDI_TRY(launch(b, 0, k_adj_blur, pb, dim3(256), 0, s, (const double *)o.tmp, o.T, c, F, 1));
    TDI_CUDA(cudaMemsetAsync(o.loss, 0, F * sizeof(double), s));
    return TDI_OK;
}

tdi_status tdi_batch_loss(tdi_batch *b, const tdi_fit_config *cfg, const float *x, const float *lam, const float *L,
                          double *loss, void *stream)
{
    if (!b || !cfg || !x || !lam || !L || !loss) return fail(TDI_ERR_INVALID, "null argument");
    if (b->d.F <= 0) return fail(TDI_ERR_INVALID, "no frames: call tdi_batch_set_frames first");
    cudaStream_t s = (cudaStream_t)stream;
    AdjBufs o;
    TDI_TRY(adj_forward(b, to_cfg(*cfg), x, lam, L, s, o));
    const int F = b->d.F;
    TDI_TRY(launch(b, 0, k_adj_grad, dim3(16, F), dim3(AD_THREADS), 0, s, (const DBatch)b->d, F, (const double *)o.B,
                   (const double *)o.T, o.loss, (const double *)nullptr, (double *)nullptr));
    TDI_CUDA(cudaMemcpyAsync(loss, o.loss, F * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return TDI_OK;
}

tdi_status tdi_batch_loss_backward(tdi_batch *b, const tdi_fit_config *cfg, const float *x, const float *lam,
                                   const float *L, const double *gloss, double *gx, double *glam, double *gL,
                                   void *stream)
{
    if (!b || !cfg || !x || !lam || !L || !gloss || !gx) return fail(TDI_ERR_INVALID, "null argument");
    if (b->d.F <= 0) return fail(TDI_ERR_INVALID, "no frames: call tdi_batch_set_frames first");
    cudaStream_t s = (cudaStream_t)stream;
    const DModel &m = b->m->d;
    const Cfg c = to_cfg(*cfg);
    AdjBufs o;
    TDI_TRY(adj_forward(b, c, x, lam, L, s, o));   // recomputed: nothing is kept from the forward call
    const int F = b->d.F;
    const size_t np = (size_t)F * NPIX;
    const dim3 pb((unsigned)((np + 255) / 256));
    TDI_CUDA(cudaMemsetAsync(o.adjB, 0, np * sizeof(double), s));
    TDI_CUDA(cudaMemsetAsync(o.dP0, 0, (size_t)F * m.V * 3 * sizeof(double), s));
    TDI_CUDA(cudaMemsetAsync(o.dpos, 0, (size_t)F * m.V * 2 * sizeof(double), s));
    TDI_CUDA(cudaMemsetAsync(o.glob, 0, (size_t)F * AD_GLOB * sizeof(double), s));
    TDI_CUDA(cudaMemsetAsync(o.geps, 0, (size_t)F * m.K * sizeof(double), s));
    TDI_TRY(launch(b, 0, k_adj_grad, dim3(16, F), dim3(AD_THREADS), 0, s, (const DBatch)b->d, F, (const double *)o.B,
                   (const double *)o.T, o.loss, gloss, o.adjB));
    // transposed blur: the column pass first, then the row pass
    TDI_TRY(launch(b, 0, k_adj_blur, pb, dim3(256), 0, s, (const double *)o.adjB, o.tmp, c, F, 1));
    TDI_TRY(launch(b, 0, k_adj_blur, pb, dim3(256), 0, s, (const double *)o.tmp, o.adjI, c, F, 0));
    TDI_TRY(launch(b, 0, k_adj_frag_back, dim3(16, F), dim3(AD_THREADS), 0, s, m, (const DBatch)b->d, x, lam, L, F,
                   (const double *)o.geo, (const double *)o.R, (const double *)o.adjI, o.dP0, o.dpos, o.glob));
    TDI_TRY(launch(b, 0, k_adj_vertex_back, dim3((m.V + 255) / 256, F), dim3(256), 0, s, m, F, (const double *)o.geo,
                   (const double *)o.R, (const float *)b->d.cam, (const double *)o.dpos, o.dP0, o.glob));
    TDI_TRY(launch(b, 0, k_adj_eps, dim3((m.V + AD_VT - 1) / AD_VT, (F + AE_F - 1) / AE_F), dim3(128), 0, s, m, F, (const double *)o.dP0,
                   o.geps));
    TDI_TRY(launch(b, 0, k_adj_final, dim3((F + 127) / 128), dim3(128), 0, s, m, F, (const double *)o.R,
                   (const double *)o.glob, (const double *)o.geps, gx, glam, gL));
    return TDI_OK;
}

tdi_status tdi_batch_read(tdi_batch *b, int32_t frame, int32_t what, void *dst, int64_t capacity, int64_t *count)
{
    if (!b || !dst || frame < 0 || frame >= b->d.F) return fail(TDI_ERR_INVALID, "bad read arguments");
    const DModel &m = b->m->d;
    const DBatch &d = b->d;
    FrameCtl ctl;
    TDI_CUDA(cudaDeviceSynchronize());
    TDI_CUDA(cudaMemcpy(&ctl, d.ctl + frame, sizeof(FrameCtl), cudaMemcpyDeviceToHost));
    const int64_t N = ctl.N;
    int64_t n = 0;
    auto copy_rows = [&](const void *src, size_t row_bytes, int rows, size_t src_pitch) -> tdi_status {
        if ((int64_t)(row_bytes * rows) > capacity) return fail(TDI_ERR_INVALID, "destination too small");
        TDI_CUDA(cudaMemcpy2D(dst, row_bytes, src, src_pitch, row_bytes, rows, cudaMemcpyDeviceToHost));
        return TDI_OK;
    };
    switch (what) {
    case 0:   // fragments: 16 bytes each
        TDI_TRY(copy_rows(d.frag + (size_t)frame * NMAX, sizeof(Fragment) * N, 1, sizeof(Fragment) * NMAX));
        n = N * 4;
        break;
    case 1:   // neighbours [4][N]
        TDI_TRY(copy_rows(d.nb + (size_t)frame * 4 * NMAX, sizeof(int32_t) * N, 4, sizeof(int32_t) * NMAX));
        n = N * 4;
        break;
    case 2:   // gradients [5][N]
        TDI_TRY(copy_rows(d.fgrad + (size_t)frame * 5 * NMAX, sizeof(float) * N, 5, sizeof(float) * NMAX));
        n = N * 5;
        break;
    case 3:   // jacobian [N][KT]
        TDI_TRY(copy_rows(d.J + (size_t)frame * NMAX * m.KTP, sizeof(float) * m.KT, (int)N, sizeof(float) * m.KTP));
        n = N * m.KT;
        break;
    case 4: { // H [KT][KT], g [KT], d [KT]
        const int64_t need = (int64_t)(m.KT * m.KT + 2 * m.KT) * (int64_t)sizeof(float);
        if (need > capacity) return fail(TDI_ERR_INVALID, "destination too small");
        float *o = static_cast<float *>(dst);
        TDI_CUDA(cudaMemcpy2D(o, sizeof(float) * m.KT, d.H + (size_t)frame * m.KTP * m.KTP, sizeof(float) * m.KTP,
                              sizeof(float) * m.KT, m.KT, cudaMemcpyDeviceToHost));
        TDI_CUDA(cudaMemcpy(o + m.KT * m.KT, d.g + (size_t)frame * m.KTP, sizeof(float) * m.KT, cudaMemcpyDeviceToHost));
        TDI_CUDA(cudaMemcpy(o + m.KT * m.KT + m.KT, d.d + (size_t)frame * m.KTP, sizeof(float) * m.KT, cudaMemcpyDeviceToHost));
        n = m.KT * m.KT + 2 * m.KT;
        break;
    }
    case 5:
        if (capacity < 4 * (int64_t)sizeof(double)) return fail(TDI_ERR_INVALID, "destination too small");
        TDI_CUDA(cudaMemcpy(dst, b->scalars + (size_t)frame * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost));
        n = 4;
        break;
    case 7:   // unblurred crop [NPIX], x-major
        if (capacity < (int64_t)(NPIX * sizeof(float))) return fail(TDI_ERR_INVALID, "destination too small");
        TDI_CUDA(cudaMemcpy(dst, b->target_raw + (size_t)frame * NPIX, NPIX * sizeof(float), cudaMemcpyDeviceToHost));
        n = NPIX;
        break;
    case 8: { // frame data: xl [51], yl [51], camera [4], face size, crop origin x0, y0 (floats)
        const int64_t cnt8 = 2 * NL + 4 + 3;
        if (capacity < cnt8 * (int64_t)sizeof(float)) return fail(TDI_ERR_INVALID, "destination too small");
        float *o = static_cast<float *>(dst);
        int32_t xy[2];
        TDI_CUDA(cudaMemcpy(o, d.xl + (size_t)frame * NL, NL * sizeof(float), cudaMemcpyDeviceToHost));
        TDI_CUDA(cudaMemcpy(o + NL, d.yl + (size_t)frame * NL, NL * sizeof(float), cudaMemcpyDeviceToHost));
        TDI_CUDA(cudaMemcpy(o + 2 * NL, d.cam + (size_t)frame * 4, 4 * sizeof(float), cudaMemcpyDeviceToHost));
        TDI_CUDA(cudaMemcpy(o + 2 * NL + 4, d.face_size + frame, sizeof(float), cudaMemcpyDeviceToHost));
        TDI_CUDA(cudaMemcpy(xy, d.x0y0 + 2 * (size_t)frame, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost));
        o[2 * NL + 5] = (float)xy[0];
        o[2 * NL + 6] = (float)xy[1];
        n = cnt8;
        break;
    }
    case 6: {
        if (capacity < (int64_t)(6 * (size_t)m.V * sizeof(float))) return fail(TDI_ERR_INVALID, "destination too small");
        // stored by slot; returned in the caller's vertex numbering
        std::vector<float4> g(m.V);
        std::vector<float4> pj(m.V);
        TDI_CUDA(cudaMemcpy(g.data(), d.geo + (size_t)frame * m.V, (size_t)m.V * sizeof(float4), cudaMemcpyDeviceToHost));
        TDI_CUDA(cudaMemcpy(pj.data(), d.proj + (size_t)frame * m.V, (size_t)m.V * sizeof(float4), cudaMemcpyDeviceToHost));
        float *o = static_cast<float *>(dst);
        const std::vector<int32_t> &vs = b->m->vslot;
        for (int v = 0; v < m.V; ++v) {
            const size_t sl = (size_t)vs[v];
            o[v] = g[sl].x; o[m.V + v] = g[sl].y; o[2 * (size_t)m.V + v] = g[sl].z;
            o[3 * (size_t)m.V + v] = pj[sl].x; o[4 * (size_t)m.V + v] = pj[sl].y; o[5 * (size_t)m.V + v] = pj[sl].z;
        }
        n = 6 * (int64_t)m.V;
        break;
    }
    default:
        return fail(TDI_ERR_INVALID, "unknown item");
    }
    if (count) *count = n;
    return TDI_OK;
}

tdi_status tdi_batch_raster(tdi_batch *b, int32_t frame, const float *xp, const float *yp, const float *zc,
                            int32_t x0, int32_t y0, int32_t *n_out, uint32_t *flags_out)
{
    if (!b || !xp || !yp || !zc || frame < 0 || frame >= b->d.F) return fail(TDI_ERR_INVALID, "bad raster arguments");
    const DModel &m = b->m->d;
    DBatch &d = b->d;
    std::vector<float4> pj(m.V);
    for (int v = 0; v < m.V; ++v) pj[b->m->vslot[v]] = make_float4(xp[v], yp[v], zc[v], 0.0f);
    TDI_CUDA(cudaMemcpy(d.proj + (size_t)frame * m.V, pj.data(), sizeof(float4) * m.V, cudaMemcpyHostToDevice));
    int32_t o[2] = {x0, y0};
    TDI_CUDA(cudaMemcpy((void *)(d.x0y0 + 2 * frame), o, sizeof(o), cudaMemcpyHostToDevice));
    uint32_t zero = 0;
    TDI_CUDA(cudaMemcpy(&d.ctl[frame].flags, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    TDI_CUDA(cudaMemcpy(d.act, &frame, sizeof(int32_t), cudaMemcpyHostToDevice));
    d.nact = 1;
    TDI_TRY(launch(b, 0, k_set_render, dim3(1), dim3(256), 0, (cudaStream_t)0, d, (int)frame));
    TDI_TRY(launch(b, KID_RASTER, k_raster_depth, dim3(raster_blocks(1), 1), dim3(RD_THREADS), 0, (cudaStream_t)0, m, d));
    TDI_TRY(launch(b, KID_RESOLVE, k_raster_resolve, dim3(1), dim3(RR_THREADS), 0, (cudaStream_t)0, m, d));
    TDI_CUDA(cudaDeviceSynchronize());
    FrameCtl ctl;
    TDI_CUDA(cudaMemcpy(&ctl, d.ctl + frame, sizeof(FrameCtl), cudaMemcpyDeviceToHost));
    if (n_out) *n_out = ctl.N;
    if (flags_out) *flags_out = ctl.flags;
    return TDI_OK;
}

tdi_status tdi_batch_render(tdi_batch *b, float *images, int32_t *tri_map, void *stream)
{
    if (!b) return fail(TDI_ERR_INVALID, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    const DModel &m = b->m->d;
    DBatch &d = b->d;
    Launch L{b, m, d, s, d.F};
    Cfg c{};
    c.ref_face_size = 78.0f;
    // evaluation point = x (shape-fit full evaluation), no fitting
    TDI_TRY(launch(b, 0, k_fit_begin, L.fblocks(), dim3(128), 0, s, d));
    TDI_TRY(launch(b, 0, k_stage_start, L.fblocks(), dim3(128), 0, s, m, d, c, (int)ST_RIGID));
    int n = 0;
    TDI_TRY(compact_active(b, s, &n));
    if (n > 0) {
        TDI_TRY(launch(b, 0, k_prepare, L.wblocks(), dim3(128), 0, s, m, d, (int)ST_RIGID));
        TDI_TRY(launch(b, 0, k_compact_render, dim3(1), dim3(1024), 0, s, (const DBatch)d));
        TDI_TRY(launch_vertex(b, m, d, s, n));
        TDI_TRY(launch(b, KID_RASTER, k_raster_depth, dim3(raster_blocks(n), n), dim3(RD_THREADS), 0, s, m, d));
        TDI_TRY(launch(b, KID_RESOLVE, k_raster_resolve, dim3(n), dim3(RR_THREADS), 0, s, m, d));
    }
    float *img = d.img;                                   // [F][NPIX] image, then [F][NPIX] map
    int32_t *map = reinterpret_cast<int32_t *>(d.img + (size_t)d.F * NPIX);
    TDI_TRY(launch(b, 0, k_paint, dim3(1, d.F), dim3(1024), 0, s, m, (const DBatch)d, img, map));
    if (images) TDI_CUDA(cudaMemcpyAsync(images, img, sizeof(float) * NPIX * d.F, cudaMemcpyDeviceToHost, s));
    if (tri_map) TDI_CUDA(cudaMemcpyAsync(tri_map, map, sizeof(int32_t) * NPIX * d.F, cudaMemcpyDeviceToHost, s));
    TDI_CUDA(cudaStreamSynchronize(s));
    return TDI_OK;
}

tdi_status tdi_batch_launches(tdi_batch *b, int64_t *launches)
{
    if (!b || !launches) return fail(TDI_ERR_INVALID, "null argument");
    *launches = b->launches;
    return TDI_OK;
}

tdi_status tdi_batch_profile(tdi_batch *b, int32_t kernel_id)
{
    if (!b || kernel_id < 0 || kernel_id > KID_RESOLVE) return fail(TDI_ERR_INVALID, "bad kernel id");
    for (auto &e : b->prof_events) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    b->prof_events.clear();
    b->prof_id = kernel_id;
    b->d.prof_id = kernel_id;
    TDI_CUDA(cudaMemset(b->d.prof_frames, 0, sizeof(unsigned long long)));
    return TDI_OK;
}

tdi_status tdi_batch_profile_read(tdi_batch *b, int64_t *launches, double *total_ms, int64_t *frames)
{
    if (!b) return fail(TDI_ERR_INVALID, "null batch");
    double ms = 0.0;
    for (auto &e : b->prof_events) {
        TDI_CUDA(cudaEventSynchronize(e.second));
        float t = 0.0f;
        TDI_CUDA(cudaEventElapsedTime(&t, e.first, e.second));
        ms += t;
    }
    unsigned long long fr = 0;
    TDI_CUDA(cudaMemcpy(&fr, b->d.prof_frames, sizeof(fr), cudaMemcpyDeviceToHost));
    if (launches) *launches = (int64_t)b->prof_events.size();
    if (total_ms) *total_ms = ms;
    if (frames) *frames = (int64_t)fr;
    return TDI_OK;
}

}  // extern "C"

#include "tdi_noalloc.cu"
