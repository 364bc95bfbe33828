// Pinning driver for the CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// Runs 3DI's own CUDA kernels, compiled unmodified from the reference sources
// (src/lib/funcs.cu, newfuncs.cu, rotation_header.cu; recipe: oracle/ref.mk, output
// oracle/_ref/), on inputs the tests also give the oracle, so that the oracle's restatement
// is checked against the reference itself. Only tests/ load the resulting library; the
// product (3di_b200/) never does.
//
// The host code here is this project's: it allocates the buffers the reference's Renderer and
// Optimizer would (sizes and the relative layout the kernels rely on: Nredundant = NTMP * T
// triangle slots, Nrender_estimated = 26,000 fragment rows, the contiguous gradient blocks and
// the ushort index block d_KSX of Optimizer.h:213-361) and launches the reference's kernels in
// the order and with the launch shapes of Renderer::render (renderer.cu:635-730) and
// DerivativeComputer::compute_hessian_and_gradient (derivative_computer.cu:22-164), for a
// single frame (t = 0) with identity and texture fixed (Kalpha = Kbeta = 0, the video fit's
// setting, video_from_saved_identity.cu:154-157).
//
// Inputs are checked on the host before any launch: the reference's kernels walk triangle
// bounding boxes with 16-bit counters and index 16-bit buffers, so projections must lie in
// [0, 65535) with boxes of at most 65,536 pixels, and the survivor count must stay within
// 25,600 (beyond it fill_krels2 writes past its rows). Calls outside those limits return an
// error instead of launching.
#include "funcs.h"
#include "newfuncs.h"
#include "rotation_header.h"

#include <thrust/device_ptr.h>
#include <thrust/fill.h>
#include <thrust/remove.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

// The reference's configuration globals that these sources name (config.cu defines them from
// the YAML file; none of them affects the kernels driven here).
namespace config {
int PAD_RENDERING = 1;
int PAD_SINGLE_IMAGE = 0;
int NPTS = 0;
}  // namespace config

namespace {

// Renderer's predicate for thrust::remove_if (renderer.cu:13-19; renderer.cu is not compiled
// into this library).
template <typename T>
struct slot_is_zero {
    __host__ __device__ bool operator()(T x) const { return x == 0; }
};

constexpr int NRE = (int)Nrender_estimated;   // 26,000 fragment rows (constants.h:49)
constexpr int MAX_FRAGMENTS = 25600;          // fill_krels2 writes whole 1,024-row blocks

struct Session {
    int V = 0, T = 0, K = 0, KT = 0;
    unsigned Nred = 0;
    cublasHandle_t blas = nullptr;
    // model
    ushort *tl = nullptr;                       // [3][T]
    float *tex = nullptr;                       // [V]
    float *EX = nullptr, *EY = nullptr, *EZ = nullptr;   // pitched [V][K] rows
    size_t pitch = 0;
    cudaTextureObject_t ex_tex = 0, ey_tex = 0, ez_tex = 0;
    // geometry
    float *X0 = nullptr, *Y0 = nullptr, *Z0 = nullptr, *X = nullptr, *Y = nullptr, *Z = nullptr;
    float *xp = nullptr, *yp = nullptr;
    // renderer slots (renderer.cu:44-90)
    bool *rend_flag = nullptr;
    ushort *pixel_idx = nullptr, *triangle_idx = nullptr;
    float *alphas = nullptr, *betas = nullptr, *gammas = nullptr, *Ztmp = nullptr;
    float *Zmins = nullptr;
    unsigned *redundant_idx = nullptr;
    float *REX = nullptr, *REY = nullptr, *REZ = nullptr;   // [K][Nred]
    float *texIm = nullptr, *buffer = nullptr, *target = nullptr;
    // optimizer blocks (Optimizer.h:213-361, T = 1, Kalpha = Kbeta = 0)
    float *opt = nullptr;
    float *tex_torender, *Id_, *dI_dlambda, *dI_dL, *vx, *vy, *vz, *px, *py, *pz, *inv_vz, *inv_vz2;
    float *J;          // dI_dbeta = start of the Ktotal column blocks: epsilon[K], tau[3], u[3]
    float *dgx, *dgy;  // [Ktotal][NRE]
    float *gx, *gy, *gxs, *gys;                  // followed by gx2..gys2 (reset together)
    float *gx_norm, *gy_norm, *gxs_norm, *gys_norm, *h, *hs;
    float *JTJ, *dG, *grad_corr;
    ushort *KSX = nullptr;
    ushort *ks_unsorted, *ks_left, *ks_right, *ks_above, *ks_below, *kl_rel, *kr_rel, *ka_rel, *kb_rel,
        *ks_sortidx, *ks_sortidx_sortidx, *ks_sorted, *ks_sorted_copy, *ks_sortidx_copy,
        *kl_rel_sorted, *kr_rel_sorted, *ka_rel_sorted, *kb_rel_sorted, *M0, *cumM0;
    // state
    float *R = nullptr, *dR = nullptr, *tau = nullptr, *lam = nullptr, *L = nullptr, *cam = nullptr;
    // rotation computer buffers (rotation_header.cu:204-320)
    float *rot = nullptr;
    std::vector<int32_t> tl_host;               // corners, for the host-side input check
    std::vector<void *> allocs;
};

template <typename T>
bool dalloc(Session *s, T **p, size_t n)
{
    void *q = nullptr;
    if (cudaMalloc(&q, (n ? n : 1) * sizeof(T)) != cudaSuccess) return false;
    cudaMemset(q, 0, (n ? n : 1) * sizeof(T));
    s->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return true;
}

void destroy(Session *s)
{
    if (!s) return;
    if (s->ex_tex) cudaDestroyTextureObject(s->ex_tex);
    if (s->ey_tex) cudaDestroyTextureObject(s->ey_tex);
    if (s->ez_tex) cudaDestroyTextureObject(s->ez_tex);
    for (void *p : s->allocs) cudaFree(p);
    if (s->blas) cublasDestroy(s->blas);
    delete s;
}

cudaTextureObject_t basis_texture(float *dev, size_t pitch, int K, int V)
{
    // the Renderer's expression-basis textures (renderer.cu:510-558): pitched rows of K floats,
    // one row per vertex, default (point, unnormalised, clamp) sampling
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = dev;
    rd.res.pitch2D.width = K;
    rd.res.pitch2D.height = V;
    rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
    rd.res.pitch2D.pitchInBytes = pitch;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    cudaTextureObject_t t = 0;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) return 0;
    return t;
}

bool sync_ok() { return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess; }

// Host check of the projections before the reference's raster walks them.
bool raster_inputs_ok(const Session *s, const float *xp, const float *yp)
{
    const std::vector<int32_t> &tlh = s->tl_host;
    for (int v = 0; v < s->V; ++v)
        if (!(xp[v] >= 0.0f && xp[v] < 65000.0f && yp[v] >= 0.0f && yp[v] < 65000.0f)) return false;
    for (int t = 0; t < s->T; ++t) {
        float x0 = 1e30f, x1 = -1e30f, y0 = 1e30f, y1 = -1e30f;
        for (int r = 0; r < 3; ++r) {
            const int v = tlh[(size_t)r * s->T + t];
            x0 = fminf(x0, xp[v]); x1 = fmaxf(x1, xp[v]);
            y0 = fminf(y0, yp[v]); y1 = fmaxf(y1, yp[v]);
        }
        if ((ceilf(x1) - floorf(x0)) * (ceilf(y1) - floorf(y0)) > 65536.0f) return false;
    }
    return true;
}

// Visibility as Renderer::render does it (renderer.cu:640-677). Returns the survivor count.
int run_raster(Session *s, int x0, int y0)
{
    const unsigned Nred = s->Nred;
    thrust::fill(thrust::device, s->Zmins, s->Zmins + DIMX * DIMY, std::numeric_limits<float>::max());
    const int Nksx = NRE * 19 + NTOTAL_PIXELS * 2;
    reset_ushort_array<<<(Nksx + NTHREADS - 1) / NTHREADS, NTHREADS>>>(s->KSX, Nksx);
    get_pixels_to_render<<<(s->T * NTMP + NTHREADS - 1) / NTHREADS, NTHREADS>>>(
        s->tl, s->xp, s->yp, s->rend_flag, s->pixel_idx, s->alphas, s->betas, s->gammas, s->triangle_idx,
        s->Z, s->Ztmp, (ushort)x0, (ushort)y0, s->Zmins, s->redundant_idx, s->T, Nred);
    keep_only_minZ<<<(Nred + NTHREADS - 1) / NTHREADS, NTHREADS>>>(s->Zmins, s->Ztmp, s->pixel_idx, s->redundant_idx, Nred);
    unsigned *end = thrust::remove_if(thrust::device, s->redundant_idx, s->redundant_idx + Nred, slot_is_zero<unsigned>());
    if (!sync_ok()) return -1;
    return (int)(end - s->redundant_idx);
}

// Survivors' slots and their pixel, triangle and barycentrics.
bool read_fragments(Session *s, int N, int32_t *pix, int32_t *tri, float *al, float *be, float *ga)
{
    std::vector<unsigned> idx(N);
    std::vector<ushort> p(s->Nred), t(s->Nred);
    std::vector<float> a(s->Nred), b(s->Nred), g(s->Nred);
    if (cudaMemcpy(idx.data(), s->redundant_idx, sizeof(unsigned) * N, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(p.data(), s->pixel_idx, sizeof(ushort) * s->Nred, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(t.data(), s->triangle_idx, sizeof(ushort) * s->Nred, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(a.data(), s->alphas, sizeof(float) * s->Nred, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(b.data(), s->betas, sizeof(float) * s->Nred, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(g.data(), s->gammas, sizeof(float) * s->Nred, cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    for (int n = 0; n < N; ++n) {
        const unsigned k = idx[n];
        if (pix) pix[n] = p[k];
        if (tri) tri[n] = t[k];
        if (al) al[n] = a[k];
        if (be) be[n] = b[k];
        if (ga) ga[n] = g[k];
    }
    return true;
}

}  // namespace

extern "C" {

// Session for one model: triangles [3][T] (0-based), expression basis [V][3][K], albedo [V],
// 15 blur taps. Returns NULL when the model does not fit the reference's 16-bit indices.
void *ref_create(int V, int T, int K, const int32_t *tl, const float *E, const float *tex, const float *taps)
{
    if (V <= 0 || T <= 0 || K <= 0 || V > 65535 || T > 65535 || K > 1024) return nullptr;
    Session *s = new Session();
    s->V = V; s->T = T; s->K = K; s->KT = K + 6;
    s->Nred = (unsigned)NTMP * (unsigned)T;
    const size_t Nred = s->Nred;
    bool ok = cublasCreate(&s->blas) == CUBLAS_STATUS_SUCCESS;
    ok = ok && dalloc(s, &s->tl, 3 * (size_t)T) && dalloc(s, &s->tex, V);
    ok = ok && dalloc(s, &s->X0, V) && dalloc(s, &s->Y0, V) && dalloc(s, &s->Z0, V) && dalloc(s, &s->X, V) &&
         dalloc(s, &s->Y, V) && dalloc(s, &s->Z, V) && dalloc(s, &s->xp, V) && dalloc(s, &s->yp, V);
    ok = ok && dalloc(s, &s->rend_flag, Nred) && dalloc(s, &s->pixel_idx, Nred) && dalloc(s, &s->triangle_idx, Nred) &&
         dalloc(s, &s->alphas, Nred) && dalloc(s, &s->betas, Nred) && dalloc(s, &s->gammas, Nred) &&
         dalloc(s, &s->Ztmp, Nred) && dalloc(s, &s->Zmins, NTOTAL_PIXELS) && dalloc(s, &s->redundant_idx, Nred);
    ok = ok && dalloc(s, &s->REX, (size_t)K * Nred) && dalloc(s, &s->REY, (size_t)K * Nred) && dalloc(s, &s->REZ, (size_t)K * Nred);
    ok = ok && dalloc(s, &s->texIm, NTOTAL_PIXELS) && dalloc(s, &s->buffer, NTOTAL_PIXELS) && dalloc(s, &s->target, NTOTAL_PIXELS);
    ok = ok && dalloc(s, &s->R, 9) && dalloc(s, &s->dR, 27) && dalloc(s, &s->tau, 3) && dalloc(s, &s->lam, 3) &&
         dalloc(s, &s->L, 1) && dalloc(s, &s->cam, 4) && dalloc(s, &s->rot, 3 + 3 + 18 + 9 * 11 + 27);
    // Optimizer block in the order of Optimizer.h:223-305 (one frame, no identity/texture)
    const size_t KT = s->KT;
    const size_t nopt = (size_t)NRE * (1 + 1 + 3 + 1 + 8) + KT * NRE + 2 * KT * NRE + (size_t)NRE * 8 +
                        (size_t)NRE * 6 + KT * KT + KT + 1 + (size_t)V;
    ok = ok && dalloc(s, &s->opt, nopt);
    ok = ok && dalloc(s, &s->KSX, (size_t)NRE * 19 + NTOTAL_PIXELS * 2);
    if (!ok) { destroy(s); return nullptr; }
    float *o = s->opt;
    s->tex_torender = o; o += NRE;
    s->Id_ = o; o += NRE;
    s->dI_dlambda = o; o += 3 * NRE;
    s->dI_dL = o; o += NRE;
    s->vx = o; o += NRE; s->vy = o; o += NRE; s->vz = o; o += NRE;
    s->px = o; o += NRE; s->py = o; o += NRE; s->pz = o; o += NRE;
    s->inv_vz = o; o += NRE; s->inv_vz2 = o; o += NRE;
    s->J = o; o += KT * NRE;
    s->dgx = o; o += KT * NRE; s->dgy = o; o += KT * NRE;
    s->gx = o; o += NRE; s->gy = o; o += NRE; s->gxs = o; o += NRE; s->gys = o; o += NRE;
    o += 4 * NRE;                                          // gx2, gy2, gxs2, gys2
    s->gx_norm = o; o += NRE; s->gy_norm = o; o += NRE; s->gxs_norm = o; o += NRE; s->gys_norm = o; o += NRE;
    s->h = o; o += NRE; s->hs = o; o += NRE;
    s->JTJ = o; o += KT * KT;
    s->dG = o; o += KT;
    s->grad_corr = o; o += 1;
    ushort *k = s->KSX;
    ushort **regions[18] = {&s->ks_unsorted, &s->ks_left, &s->ks_right, &s->ks_above, &s->ks_below, &s->kl_rel,
                            &s->kr_rel, &s->ka_rel, &s->kb_rel, &s->ks_sortidx, &s->ks_sortidx_sortidx, &s->ks_sorted,
                            &s->ks_sorted_copy, &s->ks_sortidx_copy, &s->kl_rel_sorted, &s->kr_rel_sorted,
                            &s->ka_rel_sorted, &s->kb_rel_sorted};
    for (int r = 0; r < 18; ++r) *regions[r] = k + (size_t)NRE * r;
    s->M0 = k + (size_t)NRE * 18;
    s->cumM0 = s->M0 + NTOTAL_PIXELS;
    // model upload: 16-bit corners, pitched basis rows per coordinate
    std::vector<ushort> tl16(3 * (size_t)T);
    s->tl_host.assign(tl, tl + 3 * (size_t)T);
    for (size_t i = 0; i < tl16.size(); ++i) tl16[i] = (ushort)tl[i];
    std::vector<float> rows((size_t)V * K);
    float **dst[3] = {&s->EX, &s->EY, &s->EZ};
    for (int c = 0; c < 3 && ok; ++c) {
        for (int v = 0; v < V; ++v)
            for (int q = 0; q < K; ++q) rows[(size_t)v * K + q] = E[((size_t)v * 3 + c) * K + q];
        void *p = nullptr;
        ok = cudaMallocPitch(&p, &s->pitch, sizeof(float) * K, V) == cudaSuccess;
        if (!ok) break;
        s->allocs.push_back(p);
        *dst[c] = static_cast<float *>(p);
        ok = cudaMemcpy2D(p, s->pitch, rows.data(), sizeof(float) * K, sizeof(float) * K, V, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    ok = ok && cudaMemcpy(s->tl, tl16.data(), sizeof(ushort) * tl16.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(s->tex, tex, sizeof(float) * V, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) {
        s->ex_tex = basis_texture(s->EX, s->pitch, K, V);
        s->ey_tex = basis_texture(s->EY, s->pitch, K, V);
        s->ez_tex = basis_texture(s->EZ, s->pitch, K, V);
        ok = s->ex_tex && s->ey_tex && s->ez_tex;
    }
    if (ok) {
        std::vector<float> kern(taps, taps + KERNEL_LENGTH);
        setConvolutionKernel(kern.data());
        ok = sync_ok();
    }
    if (!ok) { destroy(s); return nullptr; }
    return s;
}

void ref_destroy(void *h) { destroy(static_cast<Session *>(h)); }

// R(u) and dR/du_1..3 by fill_theta_etc (rotation_header.cu:46-151), as RotationComputer::process
// launches it. R [9] column-major, dR [3][9].
int ref_rotation(void *h, const float *u, float *R, float *dR)
{
    Session *s = static_cast<Session *>(h);
    float *b = s->rot;
    float *du = b, *theta_inv2 = b + 3, *sin_theta = b + 4, *cos_inv_sum = b + 5, *u_skew = b + 6, *unorm_skew = b + 15;
    float *m = b + 24;   // R, IR, R1a..R3c: 11 matrices
    float *Rr = m, *IR = m + 9, *R1a = m + 18, *R1b = m + 27, *R1c = m + 36, *R2a = m + 45, *R2b = m + 54,
          *R2c = m + 63, *R3a = m + 72, *R3b = m + 81, *R3c = m + 90;
    float *d1 = m + 99, *d2 = m + 108, *d3 = m + 117;
    if (cudaMemcpy(du, u, 3 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    fill_theta_etc<<<1, 1>>>(du, theta_inv2, sin_theta, cos_inv_sum, u_skew, unorm_skew, Rr, IR, R1a, R1b, R1c, R2a,
                             R2b, R2c, R3a, R3b, R3c, d1, d2, d3);
    if (!sync_ok()) return -1;
    if (cudaMemcpy(R, Rr, 9 * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(dR, d1, 27 * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    return 0;
}

// Camera transform and projection of given object points by view_transform_3d_pts_and_render_2d
// (funcs.cu:395-453). out [5][V]: X, Y, Z, xp, yp.
int ref_view_transform(void *h, const float *X0, const float *Y0, const float *Z0, const float *R, const float *tau,
                       const float *cam, float *out)
{
    Session *s = static_cast<Session *>(h);
    const int V = s->V;
    if (cudaMemcpy(s->X0, X0, sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->Y0, Y0, sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->Z0, Z0, sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->R, R, 9 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->tau, tau, 3 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->cam, cam, 4 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    view_transform_3d_pts_and_render_2d<<<(V + NTHREADS - 1) / NTHREADS, NTHREADS>>>(
        s->X0, s->Y0, s->Z0, s->R, s->tau, s->tau + 1, s->tau + 2, s->cam, s->cam + 1, s->cam + 2, s->cam + 3,
        s->X, s->Y, s->Z, s->xp, s->yp, V);
    if (!sync_ok()) return -1;
    float *dev[5] = {s->X, s->Y, s->Z, s->xp, s->yp};
    for (int q = 0; q < 5; ++q)
        if (cudaMemcpy(out + (size_t)q * V, dev[q], sizeof(float) * V, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return 0;
}

// Visibility of given projections. The session's slot buffers persist between calls, as the
// Renderer's do. Returns the survivor count N (fragments written in slot order, arrays of
// capacity cap), -1 on a CUDA error, -2 for inputs outside the checked limits.
int ref_raster(void *h, const float *xp, const float *yp, const float *Z, int x0, int y0,
               int32_t *pix, int32_t *tri, float *al, float *be, float *ga, int cap)
{
    Session *s = static_cast<Session *>(h);
    const int V = s->V;
    if (x0 < 0 || y0 < 0 || x0 > 65535 || y0 > 65535 || !raster_inputs_ok(s, xp, yp)) return -2;
    if (cudaMemcpy(s->xp, xp, sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->yp, yp, sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->Z, Z, sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    const int N = run_raster(s, x0, y0);
    if (N < 0) return N;
    if (N > cap) return -2;
    if (!read_fragments(s, N, pix, tri, al, be, ga)) return -1;
    return N;
}

// One evaluation of the image term at given geometry, as fit_3DMM_shape_rigid's
// get_obj_hessian_and_gradient_multiframe does for one frame (model_fitter.cu:21-116):
// Renderer::render, the rotated expression basis at the fragments, and
// compute_hessian_and_gradient's Jacobian, chain rule and cuBLAS products.
//   geo [8][V]: X0, Y0, Z0 (object), X, Y, Z (camera), xp, yp;  R [9], dR [3][9], tau [3],
//   lam [3], L, cam [4] (phix, phiy, cx, cy), target [65536] unblurred crop (blurred here by the
//   reference's convolution, video_fitter.cu:548-549), crop origin, tau_img (the image term's
//   log-barrier weight, 25 in the shape fit).
// Outputs (N = return value; arrays of capacity cap fragments):
//   pix, tri, al, be [N]; shade [N] (tex_torender); image [65536] (blurred render);
//   grads [7][N]: gx, gy, h, gx/|g|, gy/|g| of the render, gx/|g|, gy/|g| of the target;
//   nb [4][N]: kl, kr, ka, kb; J [N][K+6] (dI/dtheta, columns epsilon, tau, u);
//   H [(K+6)^2] (JTJ, column-major), g [K+6] (dG_dtheta); corr [1] (grad_corr = tau_img * sum).
// Returns N, -1 on a CUDA error, -2 for inputs outside the checked limits, -3 when the
// reference skips the render (N outside [1000, 52000], renderer.cu:669-677).
int ref_evaluate(void *h, const float *geo, const float *R, const float *dR, const float *tau, const float *lam,
                 float L, const float *cam, const float *target, int x0, int y0, float tau_img, int cap,
                 int32_t *pix, int32_t *tri, float *al, float *be, float *shade, float *image, float *grads,
                 int32_t *nb, float *J, float *H, float *g, float *corr)
{
    Session *s = static_cast<Session *>(h);
    const int V = s->V, K = s->K, KT = s->KT;
    const float *xp = geo + 6 * (size_t)V, *yp = geo + 7 * (size_t)V;
    if (x0 < 0 || y0 < 0 || x0 > 65535 || y0 > 65535 || !raster_inputs_ok(s, xp, yp)) return -2;
    float *dev[8] = {s->X0, s->Y0, s->Z0, s->X, s->Y, s->Z, s->xp, s->yp};
    for (int q = 0; q < 8; ++q)
        if (cudaMemcpy(dev[q], geo + (size_t)q * V, sizeof(float) * V, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    if (cudaMemcpy(s->R, R, 9 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->dR, dR, 27 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->tau, tau, 3 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->lam, lam, 3 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->L, &L, sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->target, target, sizeof(float) * NTOTAL_PIXELS, cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    // target blur (video_fitter.cu:548-549)
    convolutionRowsGPU(s->buffer, s->target, DIMX, DIMY);
    convolutionColumnsGPU(s->target, s->buffer, DIMX, DIMY);
    // Renderer::render (renderer.cu:635-730), t = 0, reset_texim = true
    cudaMemset(s->gx_norm, 0, sizeof(float) * NRE * 6);
    cudaMemset(s->texIm, 0, sizeof(float) * NTOTAL_PIXELS);
    cudaMemset(s->gx, 0, sizeof(float) * NRE * 8);
    const int N = run_raster(s, x0, y0);
    if (N < 0) return N;
    if (N > 2 * NRE || N < 1000) return -3;
    if (N > MAX_FRAGMENTS || N > cap) return -2;
    const unsigned nb_blocks = (N + NTHREADS - 1) / NTHREADS;
    fill_diffuse_component_and_populate_texture_and_shape<<<nb_blocks, NTHREADS>>>(
        s->X0, s->Y0, s->Z0, s->X, s->Y, s->Z, s->redundant_idx, s->tl, s->triangle_idx, s->alphas, s->betas,
        s->gammas, s->Ztmp, s->Id_, s->tex, s->tex_torender, s->dI_dlambda, s->dI_dL, s->vx, s->vy, s->vz, s->px,
        s->py, s->pz, s->inv_vz, s->inv_vz2, s->R, s->tau, s->lam, s->L, N, NRE, false, s->T);
    fill_ks_and_M0<<<nb_blocks, NTHREADS>>>(s->pixel_idx, s->redundant_idx, s->ks_sorted, s->ks_unsorted, s->M0, N);
    fill_tex_im1<<<nb_blocks, NTHREADS>>>(s->ks_unsorted, s->tex_torender, s->texIm, N);
    convolutionRowsGPU(s->buffer, s->texIm, DIMX, DIMY);
    convolutionColumnsGPU(s->texIm, s->buffer, DIMX, DIMY);
    fill_grads<<<nb_blocks, NTHREADS>>>(s->ks_unsorted, s->texIm, s->target, s->gx, s->gy, s->gx_norm, s->gy_norm, s->h,
                                        s->gxs, s->gys, s->gxs_norm, s->gys_norm, s->hs, N, NRE);
    const float zero = 0.0f, one = 1.0f;
    float tl_b = tau_img;
    cublasSgemm(s->blas, CUBLAS_OP_N, CUBLAS_OP_N, 1, 1, 2 * NRE, &tl_b, s->gx_norm, 1, s->gxs_norm, 2 * NRE, &zero,
                s->grad_corr, 1);
    // rotated expression basis at the fragments (model_fitter.cu:72-75)
    render_expression_basis_texture_colmajor_rotated2_via_object<<<N, K>>>(
        s->alphas, s->betas, s->gammas, s->redundant_idx, N, s->tl, s->REX, s->REY, s->REZ, s->triangle_idx, s->R, s->T,
        s->Nred, s->ex_tex, s->ey_tex, s->ez_tex);
    // DerivativeComputer::compute_hessian_and_gradient (derivative_computer.cu:38-164)
    cudaMemset(s->J, 0, sizeof(float) * KT * NRE);
    thrust::inclusive_scan(thrust::device, s->M0, s->M0 + NTOTAL_PIXELS, s->cumM0);
    thrust::sequence(thrust::device, s->ks_sortidx, s->ks_sortidx + N);
    thrust::sort_by_key(thrust::device, s->ks_sorted, s->ks_sorted + N, s->ks_sortidx);
    thrust::sequence(thrust::device, s->ks_sortidx_sortidx, s->ks_sortidx_sortidx + N);
    cudaMemcpy(s->ks_sortidx_copy, s->ks_sortidx, sizeof(ushort) * NRE, cudaMemcpyDeviceToDevice);
    thrust::sort_by_key(thrust::device, s->ks_sortidx_copy, s->ks_sortidx_copy + N, s->ks_sortidx_sortidx);
    fill_ksides<<<nb_blocks, NTHREADS>>>(s->ks_sorted, s->ks_left, s->ks_right, s->ks_above, s->ks_below);
    fill_krels<<<nb_blocks, NTHREADS>>>(N, s->ks_sorted, s->ks_sortidx, s->ks_sortidx_sortidx, s->ks_left, s->ks_right,
                                        s->ks_above, s->ks_below, s->kl_rel, s->kr_rel, s->ka_rel, s->kb_rel,
                                        s->kl_rel_sorted, s->kr_rel_sorted, s->ka_rel_sorted, s->kb_rel_sorted, s->cumM0);
    fill_krels2<<<nb_blocks, NTHREADS>>>(s->ks_unsorted, s->ks_sortidx, s->ks_sortidx_sortidx, s->kl_rel, s->kr_rel,
                                         s->ka_rel, s->kb_rel, s->kl_rel_sorted, s->kr_rel_sorted, s->ka_rel_sorted,
                                         s->kb_rel_sorted);
    float *dpose = s->J + (size_t)K * NRE;
    fill_optimization_auxiliary_variables_phase1<<<nb_blocks, NTHREADS>>>(
        cam[0], cam[1], s->vx, s->vy, s->vz, s->inv_vz, s->inv_vz2, s->px, s->py, s->pz, s->R, s->dR, s->dR + 9,
        s->dR + 18, s->gx, s->gy, dpose, dpose + NRE, dpose + 2 * NRE, dpose + 3 * NRE, dpose + 4 * NRE,
        dpose + 5 * NRE, N);
    fill_optimization_dI_depsilon_userotated<<<(N * K + NTHREADS - 1) / NTHREADS, NTHREADS>>>(
        cam[0], cam[1], s->vx, s->vy, s->vz, s->inv_vz2, s->R, s->gx, s->gy, s->REX, s->REY, s->REZ, s->J, N, K, s->Nred);
    fill_optimization_auxiliary_variables_phase2_new<<<(NRE * KT + NTHREADS - 1) / NTHREADS, NTHREADS>>>(
        s->J, s->gx, s->gy, s->h, s->kl_rel, s->kr_rel, s->ka_rel, s->kb_rel, s->dgx, s->dgy, N, KT);
    cudaMemset(s->JTJ, 0, sizeof(float) * KT * KT);
    cudaMemset(s->dG, 0, sizeof(float) * KT);
    float hb = tau_img;
    cublasSgemm(s->blas, CUBLAS_OP_T, CUBLAS_OP_N, KT, KT, NRE, &hb, s->dgx, NRE, s->dgx, NRE, &one, s->JTJ, KT);
    cublasSgemm(s->blas, CUBLAS_OP_T, CUBLAS_OP_N, KT, KT, NRE, &hb, s->dgy, NRE, s->dgy, NRE, &one, s->JTJ, KT);
    hb *= -1.0f;
    cublasSgemm(s->blas, CUBLAS_OP_N, CUBLAS_OP_N, 1, KT, NRE, &hb, s->gxs_norm, 1, s->dgx, NRE, &one, s->dG, 1);
    cublasSgemm(s->blas, CUBLAS_OP_N, CUBLAS_OP_N, 1, KT, NRE, &hb, s->gys_norm, 1, s->dgy, NRE, &one, s->dG, 1);
    if (!sync_ok()) return -1;
    // read back
    if (!read_fragments(s, N, pix, tri, al, be, nullptr)) return -1;
    bool ok = true;
    if (shade) ok = ok && cudaMemcpy(shade, s->tex_torender, sizeof(float) * N, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (image) ok = ok && cudaMemcpy(image, s->texIm, sizeof(float) * NTOTAL_PIXELS, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (grads) {
        float *src[7] = {s->gx, s->gy, s->h, s->gx_norm, s->gy_norm, s->gxs_norm, s->gys_norm};
        for (int q = 0; q < 7 && ok; ++q)
            ok = cudaMemcpy(grads + (size_t)q * N, src[q], sizeof(float) * N, cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    if (nb && ok) {
        std::vector<ushort> t(N);
        ushort *src[4] = {s->kl_rel, s->kr_rel, s->ka_rel, s->kb_rel};
        for (int q = 0; q < 4 && ok; ++q) {
            ok = cudaMemcpy(t.data(), src[q], sizeof(ushort) * N, cudaMemcpyDeviceToHost) == cudaSuccess;
            for (int n = 0; n < N; ++n) nb[(size_t)q * N + n] = t[n];
        }
    }
    if (J && ok) {
        std::vector<float> col((size_t)NRE * KT);
        ok = cudaMemcpy(col.data(), s->J, sizeof(float) * col.size(), cudaMemcpyDeviceToHost) == cudaSuccess;
        for (int n = 0; n < N; ++n)
            for (int j = 0; j < KT; ++j) J[(size_t)n * KT + j] = col[(size_t)j * NRE + n];
    }
    if (H) ok = ok && cudaMemcpy(H, s->JTJ, sizeof(float) * KT * KT, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (g) ok = ok && cudaMemcpy(g, s->dG, sizeof(float) * KT, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (corr) ok = ok && cudaMemcpy(corr, s->grad_corr, sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess;
    return ok ? N : -1;
}

}  // extern "C"
