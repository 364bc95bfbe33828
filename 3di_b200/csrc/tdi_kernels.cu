// Kernels of the batched 3DI fitting path (sm_100a). Built with -fmad=false: every formula
// below is evaluated in the operand order of the 3DI sources it restates, without FMA
// contraction, so each per-fragment quantity is bit-identical to the CPU oracle's.
#include "tdi_internal.cuh"
#include "tdi_async.cuh"

#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cfloat>
#include <cmath>

namespace tdi {

// ------------------------------------------------------------------------------------------
// Rotation R(u) and dR/du_i (rotation_header.cu:46-151).

__device__ __forceinline__ void mul33(const float *A, const float *B, float *C)
{
    C[0] = (A[0] * B[0] + A[3] * B[1]) + A[6] * B[2];
    C[1] = (A[1] * B[0] + A[4] * B[1]) + A[7] * B[2];
    C[2] = (A[2] * B[0] + A[5] * B[1]) + A[8] * B[2];
    C[3] = (A[0] * B[3] + A[3] * B[4]) + A[6] * B[5];
    C[4] = (A[1] * B[3] + A[4] * B[4]) + A[7] * B[5];
    C[5] = (A[2] * B[3] + A[5] * B[4]) + A[8] * B[5];
    C[6] = (A[0] * B[6] + A[3] * B[7]) + A[6] * B[8];
    C[7] = (A[1] * B[6] + A[4] * B[7]) + A[7] * B[8];
    C[8] = (A[2] * B[6] + A[5] * B[7]) + A[8] * B[8];
}

__device__ __forceinline__ void skew(float *S, const float *u)
{
    S[0] = 0; S[1] = u[2]; S[2] = -u[1];
    S[3] = -u[2]; S[4] = 0; S[5] = u[0];
    S[6] = u[1]; S[7] = -u[0]; S[8] = 0;
}

__device__ void rotation(const float *u, float *R, float *dR)
{
    float theta = sqrtf((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
    float un[3] = {u[0] / theta, u[1] / theta, u[2] / theta};
    float R1[3][9], Sn[9], Sn2[9];
    skew(R1[0], u); skew(R1[1], u); skew(R1[2], u);
    skew(Sn, un);
    float st = (float)sin((double)theta);
    float cis = 1.0f - (float)cos((double)theta);
    float tinv2 = 1.0f / (theta * theta);
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i < 9; ++i) R1[a][i] *= u[a];
    mul33(Sn, Sn, Sn2);
    for (int i = 0; i < 9; ++i) {
        if (i == 0 || i == 4 || i == 8)
            R[i] = (cis * Sn2[i] + 1.0f) + st * Sn[i];
        else
            R[i] = cis * Sn2[i] + st * Sn[i];
    }
    float IR[9];
    for (int i = 0; i < 9; ++i) IR[i] = R[i] * -1.0f;
    IR[0] += 1; IR[4] += 1; IR[8] += 1;
    for (int a = 0; a < 3; ++a) {
        float R2[9], R3[9];
        const float *c = IR + 3 * a;
        R2[0] = u[0] * c[0]; R2[1] = u[0] * c[1]; R2[2] = u[0] * c[2];
        R2[3] = u[1] * c[0]; R2[4] = u[1] * c[1]; R2[5] = u[1] * c[2];
        R2[6] = u[2] * c[0]; R2[7] = u[2] * c[1]; R2[8] = u[2] * c[2];
        for (int i = 0; i < 9; ++i) R1[a][i] += R2[i];
        R3[0] = R1[a][0] - R2[0]; R3[1] = R1[a][1] - R2[3]; R3[2] = R1[a][2] - R2[6];
        R3[3] = R1[a][3] - R2[1]; R3[4] = R1[a][4] - R2[4]; R3[5] = R1[a][5] - R2[7];
        R3[6] = R1[a][6] - R2[2]; R3[7] = R1[a][7] - R2[5]; R3[8] = R1[a][8] - R2[8];
        mul33(R3, R, dR + 9 * a);
        for (int i = 0; i < 9; ++i) dR[9 * a + i] *= tinv2;
    }
}

// Kernel ids for live profiling (tdi_batch_profile).
enum KernelId : int32_t { KID_VERTEX = 1, KID_RASTER = 2, KID_RENDER = 3, KID_NEIGHBOURS = 4,
                          KID_JACOBIAN = 5, KID_NORMAL_EQ = 6, KID_BARRIER = 7, KID_SOLVE = 8,
                          KID_RESOLVE = 9 };

__device__ __forceinline__ void prof_count(const DBatch &b, int id, unsigned long long n = 1)
{
    if (b.prof_id == id) atomicAdd(b.prof_frames, n);
}

// ------------------------------------------------------------------------------------------
// Stage control.

// Frames running the stage this round: the host's count, or the device count the previous
// round's compaction wrote (rounds replayed from a CUDA graph, whose grids are sized for a
// capacity; blocks past the count return at once).
__device__ __forceinline__ int active_n(const DBatch &b) { return b.dnact ? *b.dnact : b.nact; }

__device__ __forceinline__ bool shape_stage(int stage) { return stage != ST_LAMBDA; }

// Writes x_ls = x + t*d over the first n_upd entries; returns false when tau_z < 0 (the
// reference's line search then breaks without terminating, and every later outer
// iteration repeats the same trial: the frame is stuck at x, model_fitter.cu:255-259).
__device__ bool set_trial(const DModel &m, const DBatch &b, int f, int n_upd)
{
    const float *x = b.x + (size_t)f * m.KTP;
    const float *d = b.d + (size_t)f * m.KTP;
    float *xl = b.x_ls + (size_t)f * m.KTP;
    const float t = b.ctl[f].t;
    for (int a = 0; a < n_upd; ++a) xl[a] = x[a] + t * d[a];
    return !(xl[m.K + 2] < 0.0f);
}

__device__ void end_shape_stage(const Cfg &c, FrameCtl &ctl, int stage, int outer)
{
    ctl.active = 0;
    ctl.render = 0;
    ctl.need_jac = 0;
    if (stage == ST_RIGID) ctl.iters_rigid += outer; else ctl.iters_finetune += outer;
    if (stage == ST_RIGID) ctl.stage_ok = outer > c.niters_success;
}

// Line-search rejection (model_fitter.cu:325-355): shrink t, stop below the threshold,
// otherwise place the next trial.
__device__ void shape_reject(const DModel &m, const DBatch &b, const Cfg &c, int f, int stage)
{
    FrameCtl &ctl = b.ctl[f];
    const int maxit = stage == ST_RIGID ? c.max_iters_rigid : c.max_iters_finetune;
    ctl.t = ctl.t * 0.8f;
    if (ctl.t < 0.075f) {
        end_shape_stage(c, ctl, stage, ctl.outer < maxit ? ctl.outer + 1 : ctl.outer);
        return;
    }
    const int n_upd = stage == ST_FINETUNE ? m.K : m.KT;
    if (!set_trial(m, b, f, n_upd)) {
        ctl.flags |= FLAG_STUCK_NEG_TZ;
        end_shape_stage(c, ctl, stage, maxit);
    }
}

__global__ void k_stage_start(DModel m, DBatch b, Cfg c, int stage)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.F) return;
    FrameCtl &ctl = b.ctl[f];
    const bool dead = (ctl.flags & (FLAG_RENDER_SKIPPED | FLAG_OVERFLOW)) != 0;
    ctl.active = dead ? 0 : 1;
    ctl.mode = M_FULL;
    ctl.render = 0;
    ctl.need_jac = 0;
    ctl.t = 1.0f;
    ctl.inner = 0;
    ctl.outer = 1;
    if (stage == ST_LAMBDA) {
        for (int j = 0; j < 3; ++j) b.lam_ls[f * 4 + j] = b.lam[f * 4 + j];
    }
    // fit_3DMM_lambdas copies ov.betas into ov_linesearch (model_fitter.cu:991) and so
    // does fit_to_video_frame before each shape fit (video_fitter.cu:570-574); the
    // finetune keeps the line-search state the last shape fit left.
    if (stage == ST_RIGID || stage == ST_LAMBDA) {
        for (int a = 0; a < m.KT; ++a) b.x_ls[(size_t)f * m.KTP + a] = b.x[(size_t)f * m.KTP + a];
    }
}

// Evaluation point, rotation and render flag of every active frame.
__global__ void k_prepare(DModel m, DBatch b, int stage)
{
    // a warp per frame: the lanes copy the evaluation point, lane 0 forms R(u) and dR/du
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= active_n(b)) return;
    const int f = b.act[i];
    FrameCtl &ctl = b.ctl[f];
    const bool active = ctl.active != 0;
    const bool full = ctl.mode == M_FULL;
    __syncwarp();
    if (lane == 0) {
        ctl.need_jac = 0;
        if (!active) ctl.render = 0;
    }
    if (!active) return;
    const float *src = (full || stage == ST_LAMBDA) ? b.x : b.x_ls;
    float *xe = b.xe + (size_t)f * m.KTP;
    for (int a = lane; a < m.KT; a += 32) xe[a] = src[(size_t)f * m.KTP + a];
    __syncwarp();
    if (lane == 0) {
        rotation(xe + m.K + 3, b.R + f * 9, b.dR + f * 27);
        ctl.render = 1;
    }
}

// ------------------------------------------------------------------------------------------
// Vertex stage: X0 = mean + E*eps (sequential fmaf over k), camera transform and
// projection (renderer.cu:806-861, funcs.cu:395-453). A block owns 64 frames (coefficients,
// rotations, translations, cameras and render flags staged in shared memory) and walks a
// strided set of 32-vertex tiles; each tile's basis rows (32 x 3 x KP floats, contiguous in
// HBM) are brought into shared memory by the TMA engine, one bulk copy per vertex row,
// double-buffered so that the next tile streams in while this one is computed. A thread
// owns one vertex x 8 frames (24 FMA chains). geo[f][slot] = (X0, Y0, Z0, albedo);
// proj[f][slot] = (xp, yp, camera Z, 0).
// The grid is one-dimensional (about two blocks per SM) and is split on the device by the
// number of frames that render this round (known only there): ftiles frame tiles x groups
// vertex-tile stripes, so that every block has work whatever share of the active frames
// the pre-render checks rejected.

// Two IEEE fused multiply-adds in one instruction (sm_100 packed FP32): d.x = fma(a.x, b.x, c.x),
// d.y = fma(a.y, b.y, c.y), round to nearest, denormals kept -- the same results as two fmaf.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c)
{
    float2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;"
        : "=l"(reinterpret_cast<unsigned long long &>(d))
        : "l"(reinterpret_cast<const unsigned long long &>(a)), "l"(reinterpret_cast<const unsigned long long &>(b)),
          "l"(reinterpret_cast<const unsigned long long &>(c)));
    return d;
}

constexpr int VT_V = 32;                                   // vertices per tile (one per lane)
constexpr int VT_FPT = 8, VT_F = 8 * VT_FPT;               // frames per thread, per block (full rounds)
constexpr int VT_FPT_SMALL = 2;                             // frames per thread when few frames render
constexpr int VT_FR = 16;                                   // per-frame floats: R(9), tau(3), cam(4)
constexpr int VT_BLOCKS_PER_SM = 2;
constexpr int VT_WARPS = 8;                                 // computing warps; one more issues the copies
constexpr int VT_THREADS = (VT_WARPS + 1) * 32;

__host__ __device__ __forceinline__ int vt_row(int KP) { return 3 * KP + 4; }   // basis row pitch (floats)
__host__ __device__ __forceinline__ size_t vt_smem(int KP, int NF = VT_F)
{
    return ((size_t)2 * VT_V * vt_row(KP) + (size_t)NF * KP + (size_t)NF * VT_FR) * sizeof(float);
}

// A thread's FPT coefficients at one k as frame pairs (16-byte loads for 8, 8-byte for 2).
template <int FPT>
__device__ __forceinline__ void vt_load_x(float2 (&xv)[FPT / 2], const float *p)
{
    if constexpr (FPT == 8) {
        const float4 xa = *reinterpret_cast<const float4 *>(p), xb = *reinterpret_cast<const float4 *>(p + 4);
        xv[0] = make_float2(xa.x, xa.y); xv[1] = make_float2(xa.z, xa.w);
        xv[2] = make_float2(xb.x, xb.y); xv[3] = make_float2(xb.z, xb.w);
    } else {
#pragma unroll
        for (int q = 0; q < FPT / 2; ++q) xv[q] = *reinterpret_cast<const float2 *>(p + 2 * q);
    }
}

// FPT frames per computing thread, 8 FPT per block: 8 for full rounds; 2 when few frames render
// (a 64-frame tile then carries mostly idle frames through every multiply-add).
template <int FPT>
__global__ void __launch_bounds__(VT_THREADS, VT_BLOCKS_PER_SM) k_vertex_t(DModel m, DBatch b)
{
    constexpr int VT_F = 8 * FPT;              // frames of a block tile
    constexpr int VT_FPT = FPT;
    extern __shared__ __align__(16) float vsm[];
    const int KP = m.KP, K = m.K, ER = vt_row(KP);
    float *Eb = vsm;                           // [2][VT_V][ER]: basis rows of two tiles
    float *Xs = Eb + 2 * VT_V * ER;            // [KP][VT_F]: coefficients, the block's frames innermost
    float *Fs = Xs + VT_F * KP;                // [VT_F][VT_FR]
    __shared__ int s_any;
    __shared__ volatile int s_abort;
    __shared__ int s_issued;
    __shared__ int s_render[VT_F], s_frame[VT_F];
    __shared__ __align__(8) uint64_t s_full[2], s_empty[2];
    const int ntiles = (m.V + VT_V - 1) / VT_V;
    const int rc = b.rcount[0];
    const int ftiles = (rc + VT_F - 1) / VT_F;
    if (ftiles == 0) return;
    const int groups = max(1, min(ntiles, (int)gridDim.x / ftiles));
    if ((int)blockIdx.x >= ftiles * groups) return;
    const int gy = blockIdx.x / ftiles;        // vertex-tile stripe
    const int f0 = (blockIdx.x - gy * ftiles) * VT_F;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const bool producer = threadIdx.y == VT_WARPS;
    if (tid == 0) { s_any = 0; s_abort = 0; s_issued = 0; }
    __syncthreads();
    if (tid < VT_F) {
        const int ai = f0 + tid;
        const int f = ai < rc ? b.rlist[ai] : -1;
        const int r = f >= 0 && b.ctl[f].render;
        s_frame[tid] = f;
        s_render[tid] = r;
        if (r) {
            s_any = 1;
            if (gy == 0) prof_count(b, KID_VERTEX);
        }
    }
    if (tid == 0) {
        mbar_init(smem_addr(&s_full[0]), 1);
        mbar_init(smem_addr(&s_full[1]), 1);
        mbar_init(smem_addr(&s_empty[0]), VT_WARPS);
        mbar_init(smem_addr(&s_empty[1]), VT_WARPS);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (!s_any) return;
    const int rowbytes = 3 * KP * (int)sizeof(float);
    const uint32_t eb_addr = smem_addr(Eb);
    if (!producer) {
        for (int fl = threadIdx.y; fl < VT_F; fl += VT_WARPS) {
            const int f = s_frame[fl];
            const float *xr = f >= 0 ? b.xe + (size_t)f * m.KTP : nullptr;
            for (int k = threadIdx.x; k < KP; k += 32) Xs[k * VT_F + fl] = (xr && k < K) ? xr[k] : 0.0f;
            if (threadIdx.x < VT_FR) {
                const int i = threadIdx.x;
                float v = 0.0f;
                if (f >= 0) v = i < 9 ? b.R[f * 9 + i] : i < 12 ? b.xe[(size_t)f * m.KTP + K + (i - 9)] : b.cam[f * 4 + (i - 12)];
                Fs[fl * VT_FR + i] = v;
            }
        }
    } else if (threadIdx.x == 0) {
        // the first two tiles stream in while the coefficients are staged
        for (int j = 0; j < 2; ++j) {
            const int t = gy + j * groups;
            if (t >= ntiles) break;
            const int nv = min(VT_V, m.V - t * VT_V);
            const uint32_t bar = smem_addr(&s_full[j]);
            mbar_expect_tx(bar, (uint32_t)(nv * rowbytes));
            for (int r = 0; r < nv; ++r)
                bulk_g2s(eb_addr + (uint32_t)((j * VT_V + r) * ER) * 4u, m.E + (size_t)(t * VT_V + r) * 3 * KP,
                         (uint32_t)rowbytes, bar);
        }
    }
    __syncthreads();                           // coefficients staged
    if (producer) {
        if (threadIdx.x == 0) {
            // tile j into buffer j & 1 once the computing warps have released tile j - 2
            int j = 2;
            for (;; ++j) {
                const int t = gy + j * groups;
                if (t >= ntiles || s_abort) break;
                const int buf = j & 1;
                if (!mbar_wait(smem_addr(&s_empty[buf]), (uint32_t)(((j - 2) >> 1) & 1))) {
                    s_abort = 1;
                    atomicOr(b.err, 2);
                    break;
                }
                const int nv = min(VT_V, m.V - t * VT_V);
                const uint32_t bar = smem_addr(&s_full[buf]);
                mbar_expect_tx(bar, (uint32_t)(nv * rowbytes));
                for (int r = 0; r < nv; ++r)
                    bulk_g2s(eb_addr + (uint32_t)((buf * VT_V + r) * ER) * 4u, m.E + (size_t)(t * VT_V + r) * 3 * KP,
                             (uint32_t)rowbytes, bar);
            }
            s_issued = min(j, (ntiles - gy + groups - 1) / groups);
        }
    } else {
        const int vl = threadIdx.x;
        const float *xr = Xs + threadIdx.y * VT_FPT;      // this warp's frames at k: xr[k * VT_F + q]
        for (int j = 0;; ++j) {
            const int t = gy + j * groups;
            if (t >= ntiles) break;
            const int buf = j & 1;
            const int v = t * VT_V + vl;
            // the epilogue's per-vertex inputs, loaded before the wait
            float mx = 0.0f, my = 0.0f, mz = 0.0f, tx = 0.0f;
            if (v < m.V) { mx = m.mean[v]; my = m.mean[m.V + v]; mz = m.mean[2 * m.V + v]; tx = m.tex[v]; }
            const bool w = mbar_wait(smem_addr(&s_full[buf]), (uint32_t)((j >> 1) & 1));
            if (!__all_sync(0xffffffffu, w)) {
                if (threadIdx.x == 0) { s_abort = 1; atomicOr(b.err, 2); }
                break;
            }
            const float *er = Eb + (size_t)(buf * VT_V + vl) * ER;
            // Sequential fused multiply-add over k for every output (the order the oracle uses),
            // two frames per instruction: each half of fma.rn.f32x2 is an IEEE fused
            // multiply-add, so every chain rounds exactly as fmaf would.
            float2 acc[VT_FPT / 2][3];
#pragma unroll
            for (int q = 0; q < VT_FPT / 2; ++q) acc[q][0] = acc[q][1] = acc[q][2] = make_float2(0.0f, 0.0f);
            int k = 0;
            for (; k + 4 <= K; k += 4) {
                const float4 ex = *reinterpret_cast<const float4 *>(er + k);
                const float4 ey = *reinterpret_cast<const float4 *>(er + KP + k);
                const float4 ez = *reinterpret_cast<const float4 *>(er + 2 * KP + k);
                const float exv[4] = {ex.x, ex.y, ex.z, ex.w}, eyv[4] = {ey.x, ey.y, ey.z, ey.w};
                const float ezv[4] = {ez.x, ez.y, ez.z, ez.w};
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    float2 xv[VT_FPT / 2];
                    vt_load_x<VT_FPT>(xv, xr + (k + jj) * VT_F);
                    const float2 e0 = make_float2(exv[jj], exv[jj]), e1 = make_float2(eyv[jj], eyv[jj]);
                    const float2 e2 = make_float2(ezv[jj], ezv[jj]);
#pragma unroll
                    for (int q = 0; q < VT_FPT / 2; ++q) {
                        acc[q][0] = ffma2(e0, xv[q], acc[q][0]);
                        acc[q][1] = ffma2(e1, xv[q], acc[q][1]);
                        acc[q][2] = ffma2(e2, xv[q], acc[q][2]);
                    }
                }
            }
            for (; k < K; ++k) {
                const float ex = er[k], ey = er[KP + k], ez = er[2 * KP + k];
                float2 xv[VT_FPT / 2];
                vt_load_x<VT_FPT>(xv, xr + k * VT_F);
#pragma unroll
                for (int q = 0; q < VT_FPT / 2; ++q) {
                    acc[q][0] = ffma2(make_float2(ex, ex), xv[q], acc[q][0]);
                    acc[q][1] = ffma2(make_float2(ey, ey), xv[q], acc[q][1]);
                    acc[q][2] = ffma2(make_float2(ez, ez), xv[q], acc[q][2]);
                }
            }
            __syncwarp();                          // this warp is done with the buffer
            if (threadIdx.x == 0) mbar_arrive(smem_addr(&s_empty[buf]));
            if (v < m.V) {
#pragma unroll
                for (int q = 0; q < VT_FPT; ++q) {
                    const int fl = threadIdx.y * VT_FPT + q;
                    if (!s_render[fl]) continue;
                    const int f = s_frame[fl];
                    const float *R = Fs + fl * VT_FR, *tau = R + 9, *cam = R + 12;
                    const float2 *a = acc[q >> 1];
                    const float X0 = mx + ((q & 1) ? a[0].y : a[0].x);
                    const float Y0 = my + ((q & 1) ? a[1].y : a[1].x);
                    const float Z0 = mz + ((q & 1) ? a[2].y : a[2].x);
                    const float X3 = ((R[0] * X0 + R[3] * Y0) + R[6] * Z0) + tau[0];
                    const float Y3 = ((R[1] * X0 + R[4] * Y0) + R[7] * Z0) + tau[1];
                    const float Z3 = ((R[2] * X0 + R[5] * Y0) + R[8] * Z0) + tau[2];
                    b.geo[(size_t)f * m.V + v] = make_float4(X0, Y0, Z0, tx);
                    b.proj[(size_t)f * m.V + v] = make_float4((cam[0] * X3) / Z3 + cam[2], (cam[1] * Y3) / Z3 + cam[3], Z3, 0.0f);
                }
            }
        }
    }
    __syncthreads();
    if (s_abort && tid == VT_WARPS * 32) {
        // copies of the last two issued tiles may still be in flight: wait for them (bounded)
        // before the block's shared memory is released
        for (int j = max(0, s_issued - 2); j < s_issued; ++j)
            mbar_wait(smem_addr(&s_full[j & 1]), (uint32_t)((j >> 1) & 1));
    }
}

// ------------------------------------------------------------------------------------------
// Barrier objective of a state (logbarrier_initializer.cu:1921-2093 with compute_Gs :456-520):
// expression bounds, then the four landmark box constraints. Landmark 3D points are the
// vertex-stage object coordinates at the landmark vertices (same formula as the reference's
// p0L + EL*eps). One warp per frame: lanes evaluate the -log terms (FP64 log rounded to FP32),
// lane 0 sums them sequentially in FP64 in the oracle's order.

__device__ __forceinline__ void landmark_G(const DModel &m, const DBatch &b, int f, const float *x,
                                           const float *R, int i, const float *p, float G[4])
{
    const float *tau = x + m.K;
    const float *cam = b.cam + f * 4;
    const float fs = b.face_size[f];
    const float *bnd = b.bounds + (size_t)f * 4 * NL;
    const float xl = b.xl[f * NL + i], yl = b.yl[f * NL + i];
    const float p0 = p[0], p1 = p[1], p2 = p[2];
    const float r1p = (R[0] * p0 + R[3] * p1) + R[6] * p2;
    const float r2p = (R[1] * p0 + R[4] * p1) + R[7] * p2;
    const float r3p = (R[2] * p0 + R[5] * p1) + R[8] * p2;
    const float xproj = cam[0] * ((r1p + tau[0]) / (r3p + tau[2])) + cam[2];
    const float yproj = cam[1] * ((r2p + tau[1]) / (r3p + tau[2])) + cam[3];
    G[0] = 0.0f - ((xl + bnd[0 * NL + i] * fs) - xproj);
    G[1] = 0.0f - ((yl + bnd[1 * NL + i] * fs) - yproj);
    G[2] = 0.0f - ((xproj - bnd[2 * NL + i] * fs) - xl);
    G[3] = 0.0f - ((yproj - bnd[3 * NL + i] * fs) - yl);
}

// Face-size check (renderer.cu:838-857), barrier objective and the pre-render decisions of
// a trial (model_fitter.cu:237-300): tau_z, face size, NaN barrier, then -g.d < 3e-4.
// Both need only the 51 landmark vertices, so they run before the vertex stage: the landmark
// object points and projections are formed here with the vertex stage's arithmetic (the same
// values bit for bit), and a trial rejected here costs no vertex stage and no raster.
constexpr int PC_WARPS = 8;                      // frames per block (a warp each)
constexpr int PC_LM = 5;                         // per landmark: X0, Y0, Z0, xp, yp

// Shared memory of k_precheck (floats): the landmarks' basis rows (pitch 3 KP + 1, staged once
// per block for all its frames), per warp the frame's coefficients, the barrier terms and
// the landmark points.
__host__ __device__ __forceinline__ size_t precheck_smem(int K, int KP)
{
    return ((size_t)NL * (3 * KP + 1) + (size_t)PC_WARPS * (KP + 2 * K + 4 * NL + NL * PC_LM)) * sizeof(float);
}

__global__ void __launch_bounds__(PC_WARPS * 32) k_precheck(DModel m, DBatch b, Cfg c, int stage)
{
    extern __shared__ float psm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int K = m.K, KP = m.KP, EP = 3 * KP + 1;
    const int nterm = 2 * K + 4 * NL;
    float *Es = psm;                                       // [NL][EP]
    float *xs = Es + (size_t)NL * EP + (size_t)warp * KP;  // [KP] this warp's coefficients
    float *pterm = Es + (size_t)NL * EP + (size_t)PC_WARPS * KP;   // [PC_WARPS][nterm]
    float *lm = pterm + PC_WARPS * nterm + warp * NL * PC_LM;
    // the 51 landmark basis rows, once for the block's frames
    if ((int)(blockIdx.x * PC_WARPS) >= active_n(b)) return;
    for (int q = threadIdx.x; q < NL * 3 * KP; q += PC_WARPS * 32) {
        const int li = q / (3 * KP), o = q - li * 3 * KP;
        Es[li * EP + o] = m.E[(size_t)m.lis[li] * 3 * KP + o];
    }
    __syncthreads();
    const int i = blockIdx.x * PC_WARPS + warp;
    if (i >= active_n(b)) return;
    const int f = b.act[i];
    FrameCtl &ctl = b.ctl[f];
    if (!ctl.active || !ctl.render) return;
    const float *x = b.xe + (size_t)f * m.KTP;
    const float *R = b.R + f * 9;
    for (int k = lane; k < K; k += 32) xs[k] = x[k];
    __syncwarp();
    {
        const float *tau = x + K;
        const float *cam = b.cam + f * 4;
        for (int li = lane; li < NL; li += 32) {
            const int v = m.lis[li];
            const float *er = Es + li * EP;
            float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
            for (int k = 0; k < K; ++k) {
                const float xk = xs[k];
                a0 = fmaf(er[k], xk, a0);
                a1 = fmaf(er[KP + k], xk, a1);
                a2 = fmaf(er[2 * KP + k], xk, a2);
            }
            const float X0 = m.mean[v] + a0, Y0 = m.mean[m.V + v] + a1, Z0 = m.mean[2 * m.V + v] + a2;
            const float X3 = ((R[0] * X0 + R[3] * Y0) + R[6] * Z0) + tau[0];
            const float Y3 = ((R[1] * X0 + R[4] * Y0) + R[7] * Z0) + tau[1];
            const float Z3 = ((R[2] * X0 + R[5] * Y0) + R[8] * Z0) + tau[2];
            float *o = lm + li * PC_LM;
            o[0] = X0; o[1] = Y0; o[2] = Z0;
            o[3] = (cam[0] * X3) / Z3 + cam[2];
            o[4] = (cam[1] * Y3) / Z3 + cam[3];
        }
        __syncwarp();
    }
    const float d_iod = fabsf(lm[9 * PC_LM + 3] - lm[0 * PC_LM + 3]);
    const float d_lem = fabsf(lm[0 * PC_LM + 4] - lm[40 * PC_LM + 4]);
    const float d_rem = fabsf(lm[9 * PC_LM + 4] - lm[40 * PC_LM + 4]);
    const double lim = (double)c.ref_face_size * 2;
    const int face_ok = !((double)d_iod > lim || (double)d_lem > lim || (double)d_rem > lim);
    if (!shape_stage(stage)) {
        if (lane == 0) ctl.face_ok = face_ok;
        return;
    }
    float *t = pterm + warp * nterm;
    const bool ft = stage == ST_FINETUNE;
    const float *lb = m.eps_b + (ft ? 2 : 0) * m.K;
    const float *ub = m.eps_b + (ft ? 3 : 1) * m.K;
    for (int k = lane; k < m.K; k += 32) {
        const float fub = x[k] - ub[k];
        const float flb = lb[k] - x[k];
        t[2 * k] = -(float)log((double)(-flb));
        t[2 * k + 1] = -(float)log((double)(-fub));
    }
    for (int li = lane; li < NL; li += 32) {
        float G[4];
        landmark_G(m, b, f, x, R, li, lm + li * PC_LM, G);
        for (int sset = 0; sset < 4; ++sset) t[2 * m.K + sset * NL + li] = -(float)log((double)G[sset]);
    }
    __syncwarp();
    if (lane != 0) return;
    ctl.face_ok = face_ok;
    double ob = 0.0;
    for (int q = 0; q < nterm; ++q) ob += (double)t[q];
    ctl.obj_b = (float)ob;
    if (ctl.mode != M_TRIAL) return;
    if (!face_ok || isnan(ob)) {
        ctl.render = 0;
        shape_reject(m, b, c, f, stage);
        return;
    }
    if ((double)(-ctl.l2base) < 0.0003) {
        ctl.render = 0;
        const int maxit = stage == ST_RIGID ? c.max_iters_rigid : c.max_iters_finetune;
        end_shape_stage(c, ctl, stage, ctl.outer < maxit ? ctl.outer + 1 : ctl.outer);
    }
}

// ------------------------------------------------------------------------------------------
// Visibility (get_pixels_to_render + keep_only_minZ + remove_if, funcs.cu:900-1029,
// renderer.cu:650-680) in two kernels.
//
// k_raster_depth: every triangle enumerates its <= 4 fragments in bounding-box order and
// folds a 64-bit key [epoch tag | depth bits | triangle id] into the frame's z-buffer with
// atomicMin; triangles with fragments set their bit in the frame's triangle mask. The
// z-buffer does not depend on the visiting order, so triangles are visited in Morton order
// of their centroids and their corners (vertex slots) lie close in memory.
//
// k_raster_resolve, one block per frame: lists the masked triangles in ascending order
// (clearing the mask), counts the survivors of every slot row (depth equal to the pixel
// minimum), and writes them in slot order (row r, then triangle). The pixel owner is the
// minimum key (smallest triangle among depth ties). Slot 0 is dropped, as remove_if(is_zero)
// does. The epoch tag makes earlier renders' keys lose to this one's without clearing the
// z-buffer; it is cleared once the tag range is used up.

// True when alpha + beta, formed as fl(fl(na / denom) + fl(nb / denom)), is certainly above
// 1 for na, nb of denom's (nonzero) sign, so the two divisions can be skipped. With u = 2^-24:
// a finite s = fl(na + nb) beyond lim = fl(denom (1 + 16u)) gives (na + nb) / denom > 1 + 13u
// exactly, and the rounded quotients and their rounded sum then still exceed 1. Cases the bound
// cannot settle (and |denom| below 1e-30) return false and take the exact test.
__device__ __forceinline__ bool sum_exceeds_one(float na, float nb, float denom, bool dpos)
{
    constexpr float GROW = 1.0f + 16.0f * 5.9604644775390625e-8f;
    const float s = na + nb, lim = denom * GROW;
    const bool beyond = dpos ? s > lim : s < lim;
    return beyond && fabsf(denom) >= 1e-30f && fabsf(s) <= 3.4028234663852886e38f;
}

// Samples of one triangle with corners b, c, a (rows 0, 1, 2 of the triangle list) in the
// reference's order: x-major over the integer points of the bounding box, at most NTMP.
// emit(r, pix, alpha, beta) receives each, pix wrapped to 16 bits as the reference's
// ushort index is; the count is returned.
template <class Emit>
__device__ __forceinline__ int tri_samples(float bx, float by, float cx, float cy, float ax, float ay,
                                           int x0, int y0, uint32_t &flags, Emit &&emit)
{
    const float xhi = ceilf(fmaxf(fmaxf(bx, cx), ax));
    const float yhi = ceilf(fmaxf(fmaxf(by, cy), ay));
    float xlo_f = floorf(fminf(fminf(bx, cx), ax));
    float ylo_f = floorf(fminf(fminf(by, cy), ay));
    if (!(xlo_f >= 0.0f) || !(ylo_f >= 0.0f) || xhi > 65535.0f || yhi > 65535.0f) {
        flags |= FLAG_OUT_OF_DOMAIN;
        if (!(xhi <= 65535.0f && yhi <= 65535.0f)) return 0;
        xlo_f = xlo_f >= 0.0f ? xlo_f : 0.0f;
        ylo_f = ylo_f >= 0.0f ? ylo_f : 0.0f;
    }
    // A triangle whose box exceeds the whole crop only arises from a vertex near the camera
    // plane; the reference would walk the whole box. It is skipped and flagged instead.
    if ((xhi - xlo_f) * (yhi - ylo_f) > 65536.0f) {
        flags |= FLAG_OUT_OF_DOMAIN;
        return 0;
    }
    // The reference recomputes these per sample point; they do not depend on it.
    const float v0x = bx - ax, v1x = cx - ax;
    const float v0y = by - ay, v1y = cy - ay;
    const float d00 = v0x * v0x + v0y * v0y;
    const float d01 = v0x * v1x + v0y * v1y;
    const float d11 = v1x * v1x + v1y * v1y;
    const float denom = d00 * d11 - d01 * d01;
    // With a zero or NaN denominator no sample can pass (alpha, beta become inf/NaN and
    // alpha + beta <= 1 fails).
    if (!(denom > 0.0f) && !(denom < 0.0f)) return 0;
    const bool dpos = denom > 0.0f;
    int ridx = 0;
    // Boxes of at most 2 x 2 sample points (almost every triangle of a dense face mesh): the
    // same points with the same FP32 operations, evaluated without branches (the candidates'
    // products are formed once and shared, which rounds exactly as per point). Points whose
    // alpha + beta certainly exceeds 1 are dropped before the divisions; the rest take the
    // exact test in x-major order. At most 4 fragments, so the NTMP cap cannot bind.
    if (xhi - xlo_f <= 2.0f && yhi - ylo_f <= 2.0f) {
        const int xi0 = (int)xlo_f, yi0 = (int)ylo_f;
        const float xf1 = xlo_f + 1.0f, yf1 = ylo_f + 1.0f;
        // (the reference stops at the first coordinate outside the box; xf1 < xhi implies
        // xlo_f < xhi, so these select the same points)
        const bool okx[2] = {xlo_f < xhi, xf1 < xhi}, oky[2] = {ylo_f < yhi, yf1 < yhi};
        const float v2x[2] = {xlo_f - ax, xf1 - ax}, v2y[2] = {ylo_f - ay, yf1 - ay};
        float p0x[2], p1x[2], p0y[2], p1y[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            p0x[i] = v0x * v2x[i]; p1x[i] = v1x * v2x[i];
            p0y[i] = v0y * v2y[i]; p1y[i] = v1y * v2y[i];
        }
        float na[4], nb[4];
        uint32_t cand = 0;
#pragma unroll
        for (int ix = 0; ix < 2; ++ix)
#pragma unroll
            for (int iy = 0; iy < 2; ++iy) {
                const int k = 2 * ix + iy;
                const float d20 = p0x[ix] + p0y[iy];
                const float d21 = p1x[ix] + p1y[iy];
                na[k] = d11 * d20 - d01 * d21;
                nb[k] = d00 * d21 - d01 * d20;
                const bool sa = dpos ? na[k] > 0.0f : na[k] < 0.0f;
                const bool sb = dpos ? nb[k] > 0.0f : nb[k] < 0.0f;
                const bool c = okx[ix] && oky[iy] && sa && sb && !sum_exceeds_one(na[k], nb[k], denom, dpos);
                cand |= c ? (1u << k) : 0u;
            }
        while (cand) {
            const int k = __ffs(cand) - 1;
            cand &= cand - 1;
            const float nak = k == 0 ? na[0] : k == 1 ? na[1] : k == 2 ? na[2] : na[3];
            const float nbk = k == 0 ? nb[0] : k == 1 ? nb[1] : k == 2 ? nb[2] : nb[3];
            const float alpha = nak / denom;
            const float beta = nbk / denom;
            if (alpha > 0 && beta > 0 && (alpha + beta <= 1)) {
                const int px = ((yi0 + (k & 1)) - y0) + ((xi0 + (k >> 1)) - x0) * DIM;
                if (px < 0 || px >= NPIX) flags |= FLAG_OUT_OF_DOMAIN;
                emit(ridx, (uint32_t)(uint16_t)px, alpha, beta);
                ridx++;
            }
        }
        return ridx;
    }
    // Loop counters are kept as floats (integers below 2^24 are exact), which is what the
    // reference's ushort counters are converted to in every comparison and subtraction.
    int xi = (int)xlo_f;
    for (float xf = xlo_f; xf < xhi && ridx < NTMP; xf += 1.0f, ++xi) {
        const float v2x = xf - ax;
        int yi = (int)ylo_f;
        for (float yf = ylo_f; yf < yhi && ridx < NTMP; yf += 1.0f, ++yi) {
            const float v2y = yf - ay;
            const float d20 = v0x * v2x + v0y * v2y;
            const float d21 = v1x * v2x + v1y * v2y;
            // alpha = na/denom > 0 and beta = nb/denom > 0 need na, nb to have denom's sign
            // (a quotient of opposite signs, of a zero or of a NaN is not > 0): samples that
            // fail this skip the divisions; the rest take the exact test.
            const float na = d11 * d20 - d01 * d21;
            if (!(dpos ? na > 0.0f : na < 0.0f)) continue;
            const float nb = d00 * d21 - d01 * d20;
            if (!(dpos ? nb > 0.0f : nb < 0.0f)) continue;
            if (sum_exceeds_one(na, nb, denom, dpos)) continue;
            const float alpha = na / denom;
            const float beta = nb / denom;
            if (alpha > 0 && beta > 0 && (alpha + beta <= 1)) {
                const int px = (yi - y0) + (xi - x0) * DIM;
                if (px < 0 || px >= NPIX) flags |= FLAG_OUT_OF_DOMAIN;
                emit(ridx, (uint32_t)(uint16_t)px, alpha, beta);
                ridx++;
            }
        }
    }
    return ridx;
}

// Fragments of triangle idx into arrays, corners fetched through fetch(v) -> float2.
template <class Fetch>
__device__ __forceinline__ int tri_fragments_t(const DModel &m, Fetch fetch, int idx, int x0, int y0,
                                               uint16_t pix[NTMP], float al[NTMP], float be[NTMP],
                                               uint32_t &flags)
{
    const int T = m.T;
    const float2 pb = fetch(m.tl[idx]), pc = fetch(m.tl[T + idx]), pa = fetch(m.tl[2 * T + idx]);
    return tri_samples(pb.x, pb.y, pc.x, pc.y, pa.x, pa.y, x0, y0, flags,
                       [&](int r, uint32_t px, float a, float b) { pix[r] = (uint16_t)px; al[r] = a; be[r] = b; });
}

// projections as separate planes (caller-owned arrays)
__device__ __forceinline__ int tri_fragments(const DModel &m, const float *xp, const float *yp,
                                             int idx, int x0, int y0, uint16_t pix[NTMP],
                                             float al[NTMP], float be[NTMP], uint32_t &flags)
{
    return tri_fragments_t(m, [&](int v) { return make_float2(xp[v], yp[v]); }, idx, x0, y0, pix, al, be, flags);
}

// The geometry terms of a fragment's shading: unit normal of its triangle and barycentric
// point p in model coordinates, interpolated albedo t (corners b, c, a as geometry records).
__device__ __forceinline__ void shade_geometry(const float4 &gb, const float4 &gc, const float4 &ga4, float al,
                                               float be, float (&nn)[3], float (&p)[3], float &t)
{
    const float ga = (1 - al) - be;
    const float b0x = gb.x, b0y = gb.y, b0z = gb.z;
    const float c0x = gc.x, c0y = gc.y, c0z = gc.z;
    const float a0x = ga4.x, a0y = ga4.y, a0z = ga4.z;
    const float n_vx = b0x - a0x, n_vy = b0y - a0y, n_vz = b0z - a0z;
    const float n_wx = c0x - a0x, n_wy = c0y - a0y, n_wz = c0z - a0z;
    const float nrx = n_vy * n_wz - n_vz * n_wy;
    const float nry = n_vz * n_wx - n_vx * n_wz;
    const float nrz = n_vx * n_wy - n_vy * n_wx;
    const float normn = sqrtf((nrx * nrx + nry * nry) + nrz * nrz);
    nn[0] = nrx / normn; nn[1] = nry / normn; nn[2] = nrz / normn;
    p[0] = (b0x * al + c0x * be) + a0x * ga;
    p[1] = (b0y * al + c0y * be) + a0y * ga;
    p[2] = (b0z * al + c0z * be) + a0z * ga;
    t = (gb.w * al + gc.w * be) + ga4.w * ga;
}

__device__ __forceinline__ unsigned long long zkey(uint32_t tag, float Z, int tri)
{
    return ((unsigned long long)tag << (31 + TRI_BITS)) |
           ((unsigned long long)(__float_as_uint(Z) & 0x7FFFFFFFu) << TRI_BITS) |
           (unsigned long long)(uint32_t)tri;
}

__device__ __forceinline__ bool survives(unsigned long long k, uint32_t tag, uint32_t zbits)
{
    return (uint32_t)(k >> (31 + TRI_BITS)) == tag && (uint32_t)((k >> TRI_BITS) & 0x7FFFFFFFu) == zbits;
}

constexpr int RD_THREADS = 256;             // depth pass: threads per block
constexpr int RD_BLOCKS = 16;               // depth pass: blocks per frame (at least)
constexpr int RD_MAX_BLOCKS = 256;          // depth pass: blocks per frame when few frames render
constexpr int RR_THREADS = 1024;            // resolve: one block per frame
constexpr int RR_WARPS = RR_THREADS / 32;
constexpr int RR_ILP = 2;                  // resolve: listed entries per lane in flight together

__global__ void __launch_bounds__(RD_THREADS) k_raster_depth(DModel m, DBatch b)
{
    if ((int)blockIdx.y >= active_n(b)) return;
    const int f = b.act[blockIdx.y];
    const FrameCtl &ctl = b.ctl[f];
    if (!ctl.render) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) prof_count(b, KID_RASTER);
    const uint32_t tag = TAG_MAX - (ctl.epoch + 1);
    const float4 *pj = b.proj + (size_t)f * m.V;
    unsigned long long *zb = b.zbuf + (size_t)f * NPIX;
    uint32_t *mask = b.tri_mask + (size_t)f * mask_words(m.T);
    const int x0 = b.x0y0[2 * f], y0 = b.x0y0[2 * f + 1];
    const int T = m.T;
    // each block a contiguous range of the Morton order
    const int per_block = (T + gridDim.x - 1) / gridDim.x;
    const int s_begin = blockIdx.x * per_block, s_end = min(T, s_begin + per_block);
    uint32_t flags = 0;
    for (int s = s_begin + (int)threadIdx.x; s < s_end; s += RD_THREADS) {
        const int4 tq = __ldg(m.tlo4 + s);
        const int idx = tq.w;
        const float4 pb = __ldg(pj + tq.x);
        const float4 pc = __ldg(pj + tq.y);
        const float4 pa = __ldg(pj + tq.z);
        const unsigned long long key = zkey(tag, pb.z, idx);
        const int nf = tri_samples(pb.x, pb.y, pc.x, pc.y, pa.x, pa.y, x0, y0, flags,
                                   [&](int, uint32_t px, float, float) { atomicMin(zb + px, key); });
        if (nf) {
            if (!(pb.z > 0.0f)) flags |= FLAG_OUT_OF_DOMAIN;
            atomicOr(mask + (idx >> 5), 1u << (idx & 31));
        }
    }
    if (flags) atomicOr(&b.ctl[f].flags, flags);
}

// Block-wide exclusive scan of one value per thread (RR_THREADS threads); returns the
// thread's offset and writes the total to *total. Uses s_w[RR_WARPS].
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t *s_w, uint32_t *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < RR_WARPS ? s_w[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < RR_WARPS) s_w[lane] = wi - w;
        if (lane == 31) s_w[RR_WARPS] = wi;
    }
    __syncthreads();
    const uint32_t off = s_w[warp] + inc - v;
    *total = s_w[RR_WARPS];
    __syncthreads();
    return off;
}

__global__ void __launch_bounds__(RR_THREADS) k_raster_resolve(DModel m, DBatch b)
{
    if ((int)blockIdx.x >= active_n(b)) return;
    const int f = b.act[blockIdx.x];
    FrameCtl &ctl = b.ctl[f];
    if (!ctl.render) return;
    if (threadIdx.x == 0) prof_count(b, KID_RESOLVE);
    __shared__ uint32_t s_w[RR_WARPS + 1];
    __shared__ uint32_t s_cnt[RR_WARPS][NTMP];   // survivors per warp and row
    __shared__ uint32_t s_off[RR_WARPS][NTMP];   // exclusive offsets of the warps per row
    __shared__ uint32_t s_row[NTMP + 1];         // row bases; s_row[NTMP] = total
    __shared__ int s_bbox[4];
    __shared__ uint32_t s_flags;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int T = m.T;
    const uint32_t epoch = ctl.epoch + 1;
    const uint32_t tag = TAG_MAX - epoch;
    unsigned long long *zb = b.zbuf + (size_t)f * NPIX;
    uint32_t *mask = b.tri_mask + (size_t)f * mask_words(T);
    int32_t *list = b.tri_list + (size_t)f * T;
    const float4 *pj = b.proj + (size_t)f * m.V;
    const int x0 = b.x0y0[2 * f], y0 = b.x0y0[2 * f + 1];
    if (tid == 0) {
        s_flags = 0;
        s_bbox[0] = s_bbox[2] = 1 << 30;
        s_bbox[1] = s_bbox[3] = -1;
    }

    // list of the masked triangles, ascending: each thread a contiguous run of mask words
    const int W = mask_words(T);
    const int wpt = (W + RR_THREADS - 1) / RR_THREADS;
    const int w_begin = min(W, tid * wpt), w_end = min(W, w_begin + wpt);
    uint32_t nz = 0;
    for (int w = w_begin; w < w_end; ++w) nz += __popc(__ldcg(mask + w));
    uint32_t L;
    uint32_t pos = block_scan(nz, s_w, &L);
    for (int w = w_begin; w < w_end; ++w) {
        uint32_t bits = __ldcg(mask + w);
        if (bits) mask[w] = 0u;
        while (bits) {
            const int bit = __ffs(bits) - 1;
            bits &= bits - 1u;
            list[pos++] = w * 32 + bit;
        }
    }
    __syncthreads();
    // list entries per warp, contiguous; lanes take consecutive entries
    const int per_e = (int)(((L + RR_WARPS * 32 - 1) / (RR_WARPS * 32)) * 32);
    const int e_begin = min((int)L, warp * per_e);
    const int e_end = min((int)L, e_begin + per_e);

    // Survivors of every listed triangle, per slot row and warp. When the frame's per-warp,
    // per-row staging fits the gradient buffer (unused until the render), the survivors are
    // formed once here and copied to their slots after the scan; otherwise the triangles are
    // evaluated a second time in the write pass.
    Fragment *stage = reinterpret_cast<Fragment *>(b.fgrad + (size_t)f * 5 * NMAX);
    const bool one_pass = (size_t)RR_WARPS * NTMP * per_e * sizeof(Fragment) <= (size_t)5 * NMAX * sizeof(float);
    Fragment *wstage = stage + (size_t)warp * NTMP * per_e;     // [NTMP][per_e] of this warp
    int bx0 = 1 << 30, bx1 = -1, by0 = 1 << 30, by1 = -1;
    // one listed triangle: survivor flags, owners, pixels and barycentrics of its samples
    auto evaluate = [&](int e, bool (&sv)[NTMP], bool (&own)[NTMP], uint32_t (&pix)[NTMP],
                        float (&al)[NTMP], float (&be)[NTMP]) -> int {
        const int idx = __ldcg(list + e);
        const int4 tc = __ldg(m.tl4 + idx);
        const float4 pb = __ldg(pj + tc.x);
        const float4 pc = __ldg(pj + tc.y);
        const float4 pa = __ldg(pj + tc.z);
        const uint32_t zbits = __float_as_uint(pb.z) & 0x7FFFFFFFu;
        const unsigned long long mykey = zkey(tag, pb.z, idx);
        uint32_t fl2 = 0;
        tri_samples(pb.x, pb.y, pc.x, pc.y, pa.x, pa.y, x0, y0, fl2, [&](int r, uint32_t px, float a, float bb) {
            const unsigned long long k = __ldcg(zb + px);
            sv[r] = survives(k, tag, zbits) && !(r == 0 && idx == 0);
            own[r] = (k == mykey);
            pix[r] = px; al[r] = a; be[r] = bb;
        });
        return idx;
    };
    uint32_t cnt[NTMP] = {0, 0, 0, 0};
    if (one_pass) {
        // RR_ILP entries per lane and step (entries base + 32 h + lane), in phases: all their
        // triangles' corners, all sample sets, all z-buffer keys, then the survivors entry by
        // entry in entry order, so that the dependent loads of the entries overlap
        for (int base = e_begin; base < e_end; base += 32 * RR_ILP) {
            int idx[RR_ILP];
            int4 tq[RR_ILP];
            float4 pb[RR_ILP], pc[RR_ILP], pa[RR_ILP];
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) {
                const int e = base + 32 * h + lane;
                idx[h] = e < e_end ? __ldcg(list + e) : -1;
            }
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) tq[h] = __ldg(m.tl4 + (idx[h] >= 0 ? idx[h] : 0));
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) {
                pb[h] = __ldg(pj + tq[h].x);
                pc[h] = __ldg(pj + tq[h].y);
                pa[h] = __ldg(pj + tq[h].z);
            }
            uint32_t pix[RR_ILP][NTMP];
            float al[RR_ILP][NTMP], be[RR_ILP][NTMP];
            int nf[RR_ILP];
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) {
                nf[h] = 0;
                if (idx[h] >= 0) {
                    uint32_t fl2 = 0;
                    nf[h] = tri_samples(pb[h].x, pb[h].y, pc[h].x, pc[h].y, pa[h].x, pa[h].y, x0, y0, fl2,
                                        [&](int r, uint32_t px, float a, float bb) {
                                            pix[h][r] = px; al[h][r] = a; be[h][r] = bb;
                                        });
                }
            }
            unsigned long long key[RR_ILP][NTMP];
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h)
#pragma unroll
                for (int r = 0; r < NTMP; ++r) key[h][r] = r < nf[h] ? __ldcg(zb + pix[h][r]) : 0ull;
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) {
                const uint32_t zbits = __float_as_uint(pb[h].z) & 0x7FFFFFFFu;
                const unsigned long long mykey = zkey(tag, pb[h].z, idx[h]);
#pragma unroll
                for (int r = 0; r < NTMP; ++r) {
                    const bool sv = r < nf[h] && survives(key[h][r], tag, zbits) && !(r == 0 && idx[h] == 0);
                    const unsigned msk = __ballot_sync(0xffffffffu, sv);
                    if (sv) {
                        Fragment fr;
                        fr.pix_owner = pix[h][r] | (key[h][r] == mykey ? 0x80000000u : 0u);
                        fr.tri = idx[h];
                        fr.al = al[h][r];
                        fr.be = be[h][r];
                        wstage[(size_t)r * per_e + cnt[r] + __popc(msk & lt_mask)] = fr;
                        const int px = (int)(pix[h][r] >> 8), py = (int)(pix[h][r] & 255);
                        bx0 = min(bx0, px); bx1 = max(bx1, px);
                        by0 = min(by0, py); by1 = max(by1, py);
                    }
                    cnt[r] += __popc(msk);
                }
            }
        }
    } else {
        // counts only; the survivors are formed again in the write pass
        for (int base = e_begin; base < e_end; base += 32) {
            const int e = base + lane;
            bool sv[NTMP] = {false, false, false, false};
            bool own[NTMP] = {false, false, false, false};
            uint32_t pix[NTMP] = {0, 0, 0, 0};
            float al[NTMP] = {0.0f, 0.0f, 0.0f, 0.0f}, be[NTMP] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (e < e_end) evaluate(e, sv, own, pix, al, be);
#pragma unroll
            for (int r = 0; r < NTMP; ++r) cnt[r] += __popc(__ballot_sync(0xffffffffu, sv[r]));
        }
    }
    if (lane == 0)
        for (int r = 0; r < NTMP; ++r) s_cnt[warp][r] = cnt[r];
    __syncthreads();
    if (warp == 0) {
        // per row: exclusive scan over the warps (lane = warp index)
        uint32_t rowsum[NTMP];
#pragma unroll
        for (int r = 0; r < NTMP; ++r) {
            const uint32_t v = lane < RR_WARPS ? s_cnt[lane][r] : 0u;
            uint32_t inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            if (lane < RR_WARPS) s_off[lane][r] = inc - v;
            rowsum[r] = __shfl_sync(0xffffffffu, inc, 31);
        }
        if (lane == 0) {
            uint32_t acc = 0;
            for (int r = 0; r < NTMP; ++r) { s_row[r] = acc; acc += rowsum[r]; }
            s_row[NTMP] = acc;
            ctl.N = (int)min(acc, (uint32_t)NMAX);
            uint32_t fl = 0;
            if (acc > (uint32_t)NMAX) fl |= FLAG_OVERFLOW;
            if (acc < 1000u || acc > 52000u) fl |= FLAG_RENDER_SKIPPED;
            if (acc > 25600u) fl |= FLAG_OUT_OF_DOMAIN;
            s_flags = fl;
        }
    }
    __syncthreads();

    // survivors in slot order (row, then triangle)
    uint32_t wbase[NTMP];
#pragma unroll
    for (int r = 0; r < NTMP; ++r) wbase[r] = s_row[r] + s_off[warp][r];
    Fragment *out = b.frag + (size_t)f * NMAX;
    if (one_pass) {
#pragma unroll
        for (int r = 0; r < NTMP; ++r)
            for (uint32_t k = lane; k < cnt[r]; k += 32) {
                const uint32_t p = wbase[r] + k;
                if (p < (uint32_t)NMAX) out[p] = wstage[(size_t)r * per_e + k];
            }
    } else {
        uint32_t run[NTMP] = {0, 0, 0, 0};
        for (int base = e_begin; base < e_end; base += 32) {
            const int e = base + lane;
            bool sv[NTMP] = {false, false, false, false};
            bool own[NTMP] = {false, false, false, false};
            uint32_t pix[NTMP] = {0, 0, 0, 0};
            float al[NTMP] = {0.0f, 0.0f, 0.0f, 0.0f}, be[NTMP] = {0.0f, 0.0f, 0.0f, 0.0f};
            int idx = -1;
            if (e < e_end) idx = evaluate(e, sv, own, pix, al, be);
#pragma unroll
            for (int r = 0; r < NTMP; ++r) {
                const unsigned msk = __ballot_sync(0xffffffffu, sv[r]);
                if (sv[r]) {
                    const uint32_t p = wbase[r] + run[r] + __popc(msk & lt_mask);
                    if (p < (uint32_t)NMAX) {
                        Fragment fr;
                        fr.pix_owner = pix[r] | (own[r] ? 0x80000000u : 0u);
                        fr.tri = idx;
                        fr.al = al[r];
                        fr.be = be[r];
                        out[p] = fr;
                    }
                    const int px = (int)(pix[r] >> 8), py = (int)(pix[r] & 255);
                    bx0 = min(bx0, px); bx1 = max(bx1, px);
                    by0 = min(by0, py); by1 = max(by1, py);
                }
                run[r] += __popc(msk);
            }
        }
    }
    if (bx1 >= 0) {
        atomicMin(&s_bbox[0], bx0); atomicMax(&s_bbox[1], bx1);
        atomicMin(&s_bbox[2], by0); atomicMax(&s_bbox[3], by1);
    }
    __syncthreads();
    // Shading inputs of every fragment for the renders of this raster: unit normal and n . p
    // (shc), interpolated albedo (sht), formed by shade_geometry as shade() forms them, so that
    // the renders shade from coalesced records instead of gathering the triangle corners (R,
    // tau and the light enter per render). RR_ILP fragments per thread have their loads in
    // flight together. (A separate kernel of 8 blocks per frame measured slower: 38.7 us per
    // launch against the 28 us this adds to the resolve, whose other phases it overlaps.)
    if (!(s_flags & (FLAG_RENDER_SKIPPED | FLAG_OVERFLOW))) {
        const int Nf = (int)min(s_row[NTMP], (uint32_t)NMAX);
        const float4 *geo = b.geo + (size_t)f * m.V;
        float4 *shc = b.shc + (size_t)f * NMAX;
        float *sht = b.sht + (size_t)f * NMAX;
        for (int p0 = tid; p0 < Nf; p0 += RR_THREADS * RR_ILP) {
            Fragment fr[RR_ILP];
            int4 tq[RR_ILP];
            float4 gb[RR_ILP], gc[RR_ILP], ga[RR_ILP];
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) {
                const int p = p0 + h * RR_THREADS;
                fr[h] = p < Nf ? out[p] : Fragment{0u, 0, 0.0f, 0.0f};
            }
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) tq[h] = __ldg(m.tl4 + fr[h].tri);
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) {
                gb[h] = geo[tq[h].x];
                gc[h] = geo[tq[h].y];
                ga[h] = geo[tq[h].z];
            }
#pragma unroll
            for (int h = 0; h < RR_ILP; ++h) {
                const int p = p0 + h * RR_THREADS;
                if (p >= Nf) continue;
                float nn[3], pp[3], t;
                shade_geometry(gb[h], gc[h], ga[h], fr[h].al, fr[h].be, nn, pp, t);
                shc[p] = make_float4(nn[0], nn[1], nn[2], (nn[0] * pp[0] + nn[1] * pp[1]) + nn[2] * pp[2]);
                sht[p] = t;
            }
        }
    }
    if (epoch == TAG_MAX) {
        // tag range used up: the next raster starts from a cleared z-buffer
        for (int p = tid; p < NPIX; p += RR_THREADS) zb[p] = ~0ull;
    }
    if (tid == 0) {
        const uint32_t fl = s_flags;
        ctl.epoch = epoch == TAG_MAX ? 0u : epoch;
        ctl.flags |= fl;
        ctl.renders += 1;
        ctl.shade_cached = (fl & (FLAG_RENDER_SKIPPED | FLAG_OVERFLOW)) ? 0 : 1;
        for (int q = 0; q < 4; ++q) ctl.bbox[q] = s_bbox[q];
        if (s_bbox[1] >= 0 && (s_bbox[0] < 1 || s_bbox[1] > DIM - 2 || s_bbox[2] < 1 || s_bbox[3] > DIM - 2))
            ctl.flags |= FLAG_OUT_OF_DOMAIN;
        if (fl & (FLAG_RENDER_SKIPPED | FLAG_OVERFLOW)) ctl.render = 0;
    }
}

// ------------------------------------------------------------------------------------------
// Render of one frame from its fragments, one block per frame: shading
// (fill_diffuse_component_and_populate_texture_and_shape, newfuncs.cu:18-167), owners
// painted into a zeroed image (fill_tex_im1, funcs.cu:800-817), the 15-tap separable blur
// (newfuncs.cu:539-715) over the fragment box plus its 8-pixel margin (the image is zero
// outside that box, so the result equals the full-image blur there), then the
// normalised gradients of render and target at every fragment (fill_grads, funcs.cu:842-897)
// and the correlation sum.

struct Shading {
    float tex, Id, t, nn[3], p[3], v[3];
};

__device__ __forceinline__ void camera_coords(const float *R, const float *tau, float X0, float Y0,
                                              float Z0, float &X, float &Y, float &Z)
{
    X = ((R[0] * X0 + R[3] * Y0) + R[6] * Z0) + tau[0];
    Y = ((R[1] * X0 + R[4] * Y0) + R[7] * Z0) + tau[1];
    Z = ((R[2] * X0 + R[5] * Y0) + R[8] * Z0) + tau[2];
}

__device__ __forceinline__ Shading shade(const DModel &m, const float4 *geo, const Fragment &fr,
                                         const float *R, const float *tau, const float *lam,
                                         float Lint)
{
    const int4 tc = __ldg(m.tl4 + fr.tri);
    const float al = fr.al, be = fr.be, ga = (1 - fr.al) - fr.be;
    const float4 gb = geo[tc.x], gc = geo[tc.y], ga4 = geo[tc.z];
    const float b0x = gb.x, b0y = gb.y, b0z = gb.z;
    const float c0x = gc.x, c0y = gc.y, c0z = gc.z;
    const float a0x = ga4.x, a0y = ga4.y, a0z = ga4.z;
    Shading s;
    float t;
    shade_geometry(gb, gc, ga4, al, be, s.nn, s.p, t);
    const float d0 = lam[0] - tau[0], d1 = lam[1] - tau[1], d2 = lam[2] - tau[2];
    float Id = (s.nn[0] * ((R[0] * d0 + R[1] * d1) + R[2] * d2)
                + s.nn[1] * ((R[3] * d0 + R[4] * d1) + R[5] * d2))
               + s.nn[2] * ((R[6] * d0 + R[7] * d1) + R[8] * d2);
    Id = Id - ((s.nn[0] * s.p[0] + s.nn[1] * s.p[1]) + s.nn[2] * s.p[2]);
    s.t = t;
    s.tex = t + (Lint * t) * Id;
    s.Id = Id;
    float bX, bY, bZ, cX, cY, cZ, aX, aY, aZ;
    camera_coords(R, tau, b0x, b0y, b0z, bX, bY, bZ);
    camera_coords(R, tau, c0x, c0y, c0z, cX, cY, cZ);
    camera_coords(R, tau, a0x, a0y, a0z, aX, aY, aZ);
    s.v[0] = (bX * al + cX * be) + aX * ga;
    s.v[1] = (bY * al + cY * be) + aY * ga;
    s.v[2] = (bZ * al + cZ * be) + aZ * ga;
    return s;
}

// Normalised central-difference gradient of one pixel from its four neighbours as
// fill_grads forms them (index 0 past the crop border): r, l = x + 1, x - 1; d, u = y + 1, y - 1.
__device__ __forceinline__ void grad_of(float r, float l, float d, float u, float &gx, float &gy,
                                        float &h, float &gxn, float &gyn)
{
    const float a = 0.5f * (r - l);
    const float bb = 0.5f * (d - u);
    const float hh = 1e-16f + sqrtf((4 * a) * a + (4 * bb) * bb);
    gx = a; gy = bb; h = hh;
    gxn = (2.0f * a) / hh;
    gyn = (2.0f * bb) / hh;
}

__device__ __forceinline__ void neighbour_pixels(int p, int &kr, int &kl, int &kd, int &ku)
{
    const int y = p & 255, x = p >> 8;
    kr = (x < DIM - 1) ? (x + 1) * DIM + y : 0;
    kl = (x > 0) ? (x - 1) * DIM + y : 0;
    ku = (y > 0) ? x * DIM + y - 1 : 0;
    kd = (y < DIM - 1) ? x * DIM + y + 1 : 0;
}

// Region of the render: the fragment box + 8 px, or the whole crop when the fragments touch
// its border (a border pixel's neighbour is pixel 0). Blur taps are summed in ascending
// offset order with zeros outside the region (rows along y, then columns along x).
// The region buffers carry KRAD zero lines on the blurred side, so the taps need no bounds
// test: A[xl][KRAD + yl] (pitch rh + 2 KRAD) holds the shaded image and later the blurred
// one, B[KRAD + xl][yl] (pitch rh) the row pass. They live in shared memory when they fit,
// else in the frame's global buffer. Fragment gathers are issued RENDER_U at a time before
// their results are stored.

constexpr int RENDER_THREADS = 512;
constexpr int RENDER_SMEM_FLOATS = 27 * 1024;     // padded region buffers (108 KB): two blocks per SM
constexpr int RENDER_U = 2;                       // fragments whose gathers are in flight together
constexpr int RENDER_GU = 2;                      // the same in the gradient pass (8 loads each)
constexpr int RENDER_SU = 4;                      // the same when shading from the resolve's terms
constexpr int RIMG = 2 * DIM * (DIM + 2 * KRAD);  // per-frame floats of the global fallback

__host__ __device__ __forceinline__ int region_floats(int rw, int rh)
{
    return rw * (rh + 2 * KRAD) + (rw + 2 * KRAD) * rh;
}

template <bool SMEM>
__device__ __forceinline__ void render_region(const DModel &m, const DBatch &b, const Cfg &c, int stage,
                                              int f, FrameCtl &ctl, float *A, float *B, int rx0,
                                              int ry0, int rw, int rh, double *s_red)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = RENDER_THREADS / 32;
    const int N = ctl.N;
    const int ph = rh + 2 * KRAD;
    for (int i = tid; i < rw * ph; i += RENDER_THREADS) A[i] = 0.0f;
    for (int i = tid; i < KRAD * rh; i += RENDER_THREADS) { B[i] = 0.0f; B[(KRAD + rw) * rh + i] = 0.0f; }
    __syncthreads();
    const float4 *geo = b.geo + (size_t)f * m.V;
    const float *R = b.R + f * 9;
    const float *xsrc = stage == ST_LAMBDA ? b.x : b.xe;
    const float *tau = xsrc + (size_t)f * m.KTP + m.K;
    const float *lam = (stage == ST_LAMBDA && ctl.mode == M_TRIAL) ? b.lam_ls + f * 4 : b.lam + f * 4;
    const float Lint = b.Lint[f];
    const Fragment *frags = b.frag + (size_t)f * NMAX;
    auto at = [&](int p) { return ((p >> 8) - rx0) * ph + KRAD + ((p & 255) - ry0); };
    if (stage == ST_LAMBDA || ctl.shade_cached) {
        // Each fragment's unit normal, n . p and interpolated albedo depend only on the geometry
        // of the raster: the resolve forms them (shc, sht) for every raster that renders, and
        // the light fit, which moves only the light, keeps them for all its renders and for
        // k_lambda_jac (a render that finds them missing forms them itself). A render forms
        // only the rotated light R^T (lambda - tau), once, and the same FP32 operations as
        // shade(): Id = (n0 q0 + n1 q1) + n2 q2 - n.p, I = t + (L t) Id.
        float4 *shc = b.shc + (size_t)f * NMAX;
        float *sht = b.sht + (size_t)f * NMAX;
        const bool cached = ctl.shade_cached != 0;
        const float d0 = lam[0] - tau[0], d1 = lam[1] - tau[1], d2 = lam[2] - tau[2];
        const float q0 = (R[0] * d0 + R[1] * d1) + R[2] * d2;
        const float q1 = (R[3] * d0 + R[4] * d1) + R[5] * d2;
        const float q2 = (R[6] * d0 + R[7] * d1) + R[8] * d2;
        if (cached) {
            // RENDER_SU fragments per thread: each one's pixel word and shading terms are loaded
            // together (the terms are indexed by the fragment, not by its contents)
            for (int n0 = tid; n0 < N; n0 += RENDER_THREADS * RENDER_SU) {
                uint32_t po[RENDER_SU];
                float4 sn[RENDER_SU];
                float t[RENDER_SU];
#pragma unroll
                for (int u = 0; u < RENDER_SU; ++u) {
                    const int n = n0 + u * RENDER_THREADS;
                    po[u] = 0u;
                    if (n < N) {
                        po[u] = frags[n].pix_owner;
                        sn[u] = shc[n];
                        t[u] = sht[n];
                    }
                }
#pragma unroll
                for (int u = 0; u < RENDER_SU; ++u)
                    if (po[u] & 0x80000000u) {
                        const float Id = ((sn[u].x * q0 + sn[u].y * q1) + sn[u].z * q2) - sn[u].w;
                        A[at(po[u] & 0xFFFF)] = t[u] + (Lint * t[u]) * Id;
                    }
            }
        } else
        for (int n = tid; n < N; n += RENDER_THREADS) {
            const Fragment fr = frags[n];
            const Shading s = shade(m, geo, fr, R, tau, lam, Lint);
            const float4 sn = make_float4(s.nn[0], s.nn[1], s.nn[2],
                                          (s.nn[0] * s.p[0] + s.nn[1] * s.p[1]) + s.nn[2] * s.p[2]);
            const float t = s.t;
            shc[n] = sn;
            sht[n] = t;
            if (fr.pix_owner & 0x80000000u) {
                const float Id = ((sn.x * q0 + sn.y * q1) + sn.z * q2) - sn.w;
                A[at(fr.pix_owner & 0xFFFF)] = t + (Lint * t) * Id;
            }
        }
        if (tid == 0) ctl.shade_cached = 1;
    } else
    for (int n0 = tid; n0 < N; n0 += RENDER_THREADS * RENDER_U) {
        Fragment fr[RENDER_U];
#pragma unroll
        for (int u = 0; u < RENDER_U; ++u) {
            const int n = n0 + u * RENDER_THREADS;
            fr[u] = n < N ? frags[n] : Fragment{0u, 0, 0.0f, 0.0f};
        }
        float tex[RENDER_U];
        int idx[RENDER_U];
#pragma unroll
        for (int u = 0; u < RENDER_U; ++u) {
            idx[u] = -1;
            tex[u] = 0.0f;
            if (fr[u].pix_owner & 0x80000000u) {
                tex[u] = shade(m, geo, fr[u], R, tau, lam, Lint).tex;
                idx[u] = at(fr[u].pix_owner & 0xFFFF);
            }
        }
#pragma unroll
        for (int u = 0; u < RENDER_U; ++u)
            if (idx[u] >= 0) A[idx[u]] = tex[u];
    }
    __syncthreads();
    const uint32_t mgh = 0xFFFFFFFFu / (uint32_t)rh + 1u;   // i / rh = umulhi(i, mgh) for i <= 2^16
    // rows: along the contiguous (y) index
    for (int i = tid; i < rw * rh; i += RENDER_THREADS) {
        const int xl = (int)__umulhi((uint32_t)i, mgh), yl = i - xl * rh;
        const float *a = A + xl * ph + yl;               // a[KRAD + j] = A(xl, yl + j)
        float s = 0.0f;
#pragma unroll
        for (int j = -KRAD; j <= KRAD; ++j) s = s + c.taps[KRAD - j] * a[KRAD + j];
        B[(KRAD + xl) * rh + yl] = s;
    }
    __syncthreads();
    // columns: along the strided (x) index
    for (int i = tid; i < rw * rh; i += RENDER_THREADS) {
        const int xl = (int)__umulhi((uint32_t)i, mgh), yl = i - xl * rh;
        const float *bp = B + xl * rh + yl;              // bp[(KRAD + j) * rh] = B(xl + j, yl)
        float s = 0.0f;
#pragma unroll
        for (int j = -KRAD; j <= KRAD; ++j) s = s + c.taps[KRAD - j] * bp[(KRAD + j) * rh];
        A[xl * ph + KRAD + yl] = s;
    }
    __syncthreads();
    const float *tgt = b.target + (size_t)f * NPIX;
    float *fg = b.fgrad + (size_t)f * 5 * NMAX;
    double corr = 0.0;
    for (int n0 = tid; n0 < N; n0 += RENDER_THREADS * RENDER_GU) {
        int pv[RENDER_GU];
#pragma unroll
        for (int u = 0; u < RENDER_GU; ++u) {
            const int n = n0 + u * RENDER_THREADS;
            pv[u] = n < N ? (int)(frags[n].pix_owner & 0xFFFF) : -1;
        }
        float rv[RENDER_GU][4], tv[RENDER_GU][4];
#pragma unroll
        for (int u = 0; u < RENDER_GU; ++u) {
            rv[u][0] = rv[u][1] = rv[u][2] = rv[u][3] = 0.0f;
            tv[u][0] = tv[u][1] = tv[u][2] = tv[u][3] = 0.0f;
            if (pv[u] >= 0) {                  // (pixel 0 lies outside a region that is not the crop)
                int kr, kl, kd, ku;
                neighbour_pixels(pv[u], kr, kl, kd, ku);
                rv[u][0] = A[at(kr)]; rv[u][1] = A[at(kl)]; rv[u][2] = A[at(kd)]; rv[u][3] = A[at(ku)];
                tv[u][0] = tgt[kr]; tv[u][1] = tgt[kl]; tv[u][2] = tgt[kd]; tv[u][3] = tgt[ku];
            }
        }
#pragma unroll
        for (int u = 0; u < RENDER_GU; ++u) {
            if (pv[u] < 0) break;
            const int n = n0 + u * RENDER_THREADS;
            float gx, gy, h, gxn, gyn, sx, sy, sh, sxn, syn;
            grad_of(rv[u][0], rv[u][1], rv[u][2], rv[u][3], gx, gy, h, gxn, gyn);
            grad_of(tv[u][0], tv[u][1], tv[u][2], tv[u][3], sx, sy, sh, sxn, syn);
            fg[n] = gx; fg[NMAX + n] = gy; fg[2 * NMAX + n] = h;
            fg[3 * NMAX + n] = sxn; fg[4 * NMAX + n] = syn;
            corr += (double)gxn * (double)sxn + (double)gyn * (double)syn;
        }
    }
    for (int o = 16; o > 0; o >>= 1) corr += __shfl_down_sync(0xffffffffu, corr, o);
    if (lane == 0) s_red[warp] = corr;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < NW; ++w) s += s_red[w];
        ctl.corr = s;
    }
}

__global__ void __launch_bounds__(RENDER_THREADS, 2) k_render(DModel m, DBatch b, Cfg c, int stage)
{
    if ((int)blockIdx.x >= active_n(b)) return;
    const int f = b.act[blockIdx.x];
    FrameCtl &ctl = b.ctl[f];
    if (!ctl.render) return;
    if (threadIdx.x == 0) prof_count(b, KID_RENDER);
    extern __shared__ __align__(16) float rsm[];
    __shared__ double s_red[RENDER_THREADS / 32];
    const bool border = ctl.bbox[0] < 1 || ctl.bbox[1] > DIM - 2 || ctl.bbox[2] < 1 || ctl.bbox[3] > DIM - 2;
    const int rx0 = border ? 0 : max(0, ctl.bbox[0] - 8), rx1 = border ? DIM - 1 : min(DIM - 1, ctl.bbox[1] + 8);
    const int ry0 = border ? 0 : max(0, ctl.bbox[2] - 8), ry1 = border ? DIM - 1 : min(DIM - 1, ctl.bbox[3] + 8);
    const int rw = rx1 - rx0 + 1, rh = ry1 - ry0 + 1;
    if (region_floats(rw, rh) <= RENDER_SMEM_FLOATS) {
        render_region<true>(m, b, c, stage, f, ctl, rsm, rsm + rw * (rh + 2 * KRAD), rx0, ry0, rw, rh, s_red);
    } else {
        float *g = b.img + (size_t)f * RIMG;
        render_region<false>(m, b, c, stage, f, ctl, g, g + rw * (rh + 2 * KRAD), rx0, ry0, rw, rh, s_red);
    }
}

// ------------------------------------------------------------------------------------------
// Decisions after a render.

// Shape fits (model_fitter.cu:215-356): objective -(tau*corr - barrier); Armijo test.
__global__ void k_decide_shape(DModel m, DBatch b, Cfg c, int stage)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active_n(b)) return;
    const int f = b.act[i];
    FrameCtl &ctl = b.ctl[f];
    if (!ctl.active) return;
    const int maxit = stage == ST_RIGID ? c.max_iters_rigid : c.max_iters_finetune;
    if (ctl.flags & (FLAG_RENDER_SKIPPED | FLAG_OVERFLOW)) {
        end_shape_stage(c, ctl, stage, ctl.outer);
        return;
    }
    if (!ctl.render) return;
    const float tau_img = 5.0f * 5.0f;
    float gc = tau_img * (float)ctl.corr;
    gc = gc + (-ctl.obj_b);
    const float obj = -gc;
    if (ctl.mode == M_FULL) {
        ctl.obj0 = obj;
        ctl.objective = obj;
        ctl.need_jac = 1;
        return;
    }
    ctl.inner++;
    float l2 = ctl.l2base;
    l2 = l2 * (0.4f * ctl.t);
    if (obj < ctl.obj0 + l2) {
        for (int a = 0; a < m.KT; ++a) b.x[(size_t)f * m.KTP + a] = b.x_ls[(size_t)f * m.KTP + a];
        ctl.obj0 = obj;
        ctl.objective = obj;
        if (ctl.outer >= maxit) { end_shape_stage(c, ctl, stage, ctl.outer); return; }
        ctl.outer++;
        ctl.need_jac = 1;
    } else {
        shape_reject(m, b, c, f, stage);
    }
}

// Light fit (model_fitter.cu:981-1073): objective -corr; Armijo test with alpha = beta = 0.5.
__global__ void k_decide_lambda(DModel m, DBatch b, Cfg c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active_n(b)) return;
    const int f = b.act[i];
    FrameCtl &ctl = b.ctl[f];
    if (!ctl.active) return;
    if (ctl.flags & (FLAG_RENDER_SKIPPED | FLAG_OVERFLOW)) { ctl.active = 0; return; }
    if (!ctl.render) return;
    const float obj = -(float)ctl.corr;
    if (ctl.mode == M_FULL) {
        ctl.obj0 = obj;
        ctl.iters_lambda++;
        ctl.need_jac = 1;
        return;
    }
    ctl.inner++;
    float l2 = ctl.l2base;
    l2 = l2 * (0.5f * ctl.t);
    if (obj < ctl.obj0 + l2) {
        for (int j = 0; j < 3; ++j) b.lam[f * 4 + j] = b.lam_ls[f * 4 + j];
        ctl.obj0 = obj;
        if (ctl.iters_lambda >= c.max_iters_lambda) { ctl.active = 0; return; }
        ctl.iters_lambda++;
        ctl.need_jac = 1;
    } else {
        ctl.t = ctl.t * 0.5f;
        if (ctl.t < 0.01f) { ctl.active = 0; return; }
        for (int j = 0; j < 3; ++j) b.lam_ls[f * 4 + j] = b.lam[f * 4 + j] + ctl.t * b.dlam[f * 4 + j];
    }
}

// ------------------------------------------------------------------------------------------
// Neighbour maps (derivative_computer.cu:43-72; funcs.cu:81-131, 288-343), one block per
// frame. The reference stable-sorts fragments by pixel and derives, for sorted position i,
// left = i - (cum[p] - cum[p-256]) (0 when not positive, clamped to N-1),
// right = i + cum[p+256] - cum[p], above/below = i -+ 1 (16-bit wrap), position 0 and N-1
// all 0, where cum counts distinct covered pixels up to a pixel. Here the sort is replaced by
// a counting placement: sorted position = distinct pixels below p + extra (tied) fragments
// below p + rank among the fragments of p in slot order.
// The counting atomics also build the per-word masks (covered pixels, pixels with 2+
// fragments) and extra-fragment counts, so only 2,048 words are scanned. Sorted positions
// and the inverse permutation are held in shared memory as 16-bit indices (NMAX = 32768).
// A pixel hit by several fragments (rare) first gets its fragments placed in arbitrary order
// inside its group, then each of them counts the group members with a lower slot index,
// which gives the stable order; frames without such pixels skip those passes.

constexpr int NB_U = 4;                 // fragment pixels loaded per thread before use
__host__ __device__ constexpr size_t neigh_smem()
{
    return (size_t)(NPIX / 2 + 4 * (NPIX / 32)) * sizeof(uint32_t) + (size_t)NMAX * sizeof(uint16_t);
}

__device__ __forceinline__ uint32_t cnt_at(const uint32_t *cnt, int p)
{
    return (cnt[p >> 1] >> ((p & 1) * 16)) & 0xFFFFu;
}

__global__ void __launch_bounds__(1024) k_neighbours(DBatch b, int all_frames)
{
    if ((int)blockIdx.x >= active_n(b)) return;
    const int f = b.act[blockIdx.x];
    FrameCtl &ctl = b.ctl[f];
    if (!(all_frames ? ctl.render : ctl.need_jac)) return;
    if (threadIdx.x == 0) prof_count(b, KID_NEIGHBOURS);
    extern __shared__ __align__(16) uint32_t nsm[];
    uint32_t *cnt = nsm;                    // 32768 words: two 16-bit counts each
    uint16_t *perm = reinterpret_cast<uint16_t *>(nsm);   // replaces cnt: sorted position -> fragment
    uint32_t *bits = cnt + NPIX / 2;        // 2048 words: covered pixels
    uint32_t *tieb = bits + NPIX / 32;      // 2048 words: pixels with 2+ fragments
    uint32_t *wU = tieb + NPIX / 32;        // 2048: distinct pixels before the word
    uint32_t *wE = wU + NPIX / 32;          // 2048: extra fragments in (then before) the word
    uint16_t *spos = reinterpret_cast<uint16_t *>(wE + NPIX / 32);   // [NMAX]: fragment -> sorted position
    __shared__ uint32_t s_wsum[2][32];
    __shared__ uint32_t s_flags;
    __shared__ int s_ties;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int N = ctl.N;
    const Fragment *frags = b.frag + (size_t)f * NMAX;
    auto pix_of = [&](int n) -> int { return (int)(frags[n].pix_owner & 0xFFFF); };
    auto load_pix = [&](int n0, int pv[NB_U]) {
#pragma unroll
        for (int u = 0; u < NB_U; ++u) {
            const int n = n0 + u * 1024;
            pv[u] = n < N ? pix_of(n) : 0;
        }
    };
    if (tid == 0) { s_flags = 0; s_ties = 0; }
    {
        uint4 *z = reinterpret_cast<uint4 *>(nsm);          // cnt, bits, tieb
        for (int i = tid; i < (NPIX / 2 + 2 * (NPIX / 32)) / 4; i += 1024) z[i] = make_uint4(0u, 0u, 0u, 0u);
        for (int i = tid; i < NPIX / 32; i += 1024) wE[i] = 0;
    }
    __syncthreads();
    for (int n0 = tid; n0 < N; n0 += 1024 * NB_U) {
        int pv[NB_U];
        load_pix(n0, pv);
#pragma unroll
        for (int u = 0; u < NB_U; ++u) {
            if (n0 + u * 1024 >= N) break;
            const int p = pv[u], w = p >> 5;
            const uint32_t bm = 1u << (p & 31), sh = (p & 1) * 16;
            const uint32_t old = (atomicAdd(&cnt[p >> 1], 1u << sh) >> sh) & 0xFFFFu;
            if (old == 0) {
                atomicOr(&bits[w], bm);
            } else {
                atomicAdd(&wE[w], 1u);
                if (old == 1) { atomicOr(&tieb[w], bm); s_ties = 1; }
            }
        }
    }
    __syncthreads();
    // exclusive scans of the distinct and extra counts over the 2048 words
    uint32_t u2[2], e2[2];
    for (int q = 0; q < 2; ++q) { u2[q] = __popc(bits[tid * 2 + q]); e2[q] = wE[tid * 2 + q]; }
    uint32_t us = u2[0] + u2[1], es = e2[0] + e2[1];
    uint32_t ui = us, ei = es;   // inclusive warp scans
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t a = __shfl_up_sync(0xffffffffu, ui, o), c2 = __shfl_up_sync(0xffffffffu, ei, o);
        if (lane >= o) { ui += a; ei += c2; }
    }
    if (lane == 31) { s_wsum[0][warp] = ui; s_wsum[1][warp] = ei; }
    __syncthreads();                       // also orders every read of wE above before its rewrite
    if (tid < 32) {
        uint32_t a = s_wsum[0][tid], c2 = s_wsum[1][tid];
        uint32_t ai = a, ci = c2;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t1 = __shfl_up_sync(0xffffffffu, ai, o), t2 = __shfl_up_sync(0xffffffffu, ci, o);
            if (tid >= o) { ai += t1; ci += t2; }
        }
        s_wsum[0][tid] = ai - a;
        s_wsum[1][tid] = ci - c2;
    }
    __syncthreads();
    {
        const uint32_t ubase = s_wsum[0][warp] + ui - us, ebase = s_wsum[1][warp] + ei - es;
        wU[tid * 2] = ubase; wE[tid * 2] = ebase;
        wU[tid * 2 + 1] = ubase + u2[0]; wE[tid * 2 + 1] = ebase + e2[0];
    }
    __syncthreads();
    const bool ties = s_ties != 0;
    auto cum = [&](int p) -> int {                     // covered pixels q <= p
        const int w = p >> 5, bit = p & 31;
        return (int)(wU[w] + __popc(bits[w] & ((2u << bit) - 1u)));
    };
    auto tied = [&](int p) -> bool { return (tieb[p >> 5] >> (p & 31)) & 1u; };
    // first sorted position of pixel p's fragments
    auto group_start = [&](int p) -> int {
        const int w = p >> 5;
        const uint32_t below = (1u << (p & 31)) - 1u;
        uint32_t pos = wU[w] + __popc(bits[w] & below) + wE[w];
        uint32_t tb = tieb[w] & below;
        while (tb) {
            const int j = __ffs(tb) - 1;
            tb &= tb - 1;
            pos += cnt_at(cnt, w * 32 + j) - 1;
        }
        return (int)pos;
    };
    for (int n0 = tid; n0 < N; n0 += 1024 * NB_U) {
        int pv[NB_U];
        load_pix(n0, pv);
#pragma unroll
        for (int u = 0; u < NB_U; ++u) {
            const int n = n0 + u * 1024;
            if (n < N) spos[n] = (uint16_t)group_start(pv[u]);
        }
    }
    if (ties) {
        // distinct slots inside each group, in arbitrary order: the counts are taken back one
        // by one (nothing reads them after the barrier)
        __syncthreads();
        for (int n = tid; n < N; n += 1024) {
            const int p = pix_of(n);
            if (!tied(p)) continue;
            const uint32_t sh = (p & 1) * 16;
            const uint32_t old = (atomicSub(&cnt[p >> 1], 1u << sh) >> sh) & 0xFFFFu;
            spos[n] = (uint16_t)(spos[n] + old - 1);
        }
    }
    __syncthreads();                       // the counts are no longer read: perm replaces them
    for (int n = tid; n < N; n += 1024) perm[spos[n]] = (uint16_t)n;
    __syncthreads();
    if (ties) {
        // stable order inside each group: rank = group members with a lower slot index
        for (int n = tid; n < N; n += 1024) {
            const int p = pix_of(n);
            if (!tied(p)) continue;
            const int i = spos[n];
            int r = 0, j = i - 1;
            for (; j >= 0; --j) {
                const int q = perm[j];
                if (pix_of(q) != p) break;
                r += q < n;
            }
            const int start = j + 1;
            for (j = i + 1; j < N; ++j) {
                const int q = perm[j];
                if (pix_of(q) != p) break;
                r += q < n;
            }
            spos[n] = (uint16_t)(start + r);
        }
        __syncthreads();
        for (int n = tid; n < N; n += 1024)
            if (tied(pix_of(n))) perm[spos[n]] = (uint16_t)n;
        __syncthreads();
    }
    int32_t *nb = b.nb + (size_t)f * 4 * NMAX;
    for (int n0 = tid; n0 < N; n0 += 1024 * NB_U) {
        int pv[NB_U];
        load_pix(n0, pv);
#pragma unroll
        for (int u = 0; u < NB_U; ++u) {
            const int n = n0 + u * 1024;
            if (n >= N) continue;
            const int i = spos[n], p = pv[u];
            int S[4] = {0, 0, 0, 0};
            if (i != 0 && i != N - 1) {
                const int y = p & 255, x = p >> 8;
                const int right = (x < DIM - 1) ? (x + 1) * DIM + y : 0;
                const int left = (x > 0) ? (x - 1) * DIM + y : 0;
                const int dl = cum(p) - cum(left);
                int kl = (i > dl) ? (i - dl) : 0;
                kl = (uint16_t)kl;
                if (kl >= N - 1) kl = N - 1;
                S[0] = kl;
                S[1] = (uint16_t)(i + cum(right) - cum(p));
                S[2] = (uint16_t)(i - 1);
                S[3] = (uint16_t)(i + 1);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                int sq = S[q];
                if (sq >= N) { atomicOr(&s_flags, FLAG_OUT_OF_DOMAIN); sq = 0; }
                nb[q * NMAX + n] = perm[sq];
            }
        }
    }
    __syncthreads();
    if (tid == 0 && s_flags) ctl.flags |= s_flags;
}

// ------------------------------------------------------------------------------------------
// Jacobian rows dI/dtheta (newfuncs.cu:173-299, funcs.cu:224-282). A block takes chunks of
// JAC_CH fragments of one frame: one thread per fragment forms the interpolated point, its
// camera coordinates and the pose columns, and leaves the per-fragment factors in shared
// memory; then the chunk's (fragment, expression column) items are spread over all threads,
// consecutive items being consecutive columns of a fragment, so that the three basis rows
// are read coalesced and no lane idles on a short last pass. (Taking the chunks in pixel
// order, so that a chunk's triangles share corners, measured 3% slower.)

constexpr int JAC_THREADS = 256;
constexpr int JAC_CH = 128;                  // fragments per chunk
constexpr int JAC_BPF = 32;                  // blocks per frame

__global__ void __launch_bounds__(JAC_THREADS, 4) k_jacobian(DModel m, DBatch b)
{
    if ((int)blockIdx.y >= active_n(b)) return;
    const int f = b.act[blockIdx.y];
    const FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) prof_count(b, KID_JACOBIAN);
    __shared__ float4 s_w[JAC_CH];           // al, be, ga, gx
    __shared__ float4 s_v[JAC_CH];           // vx, vy, vz, gy
    __shared__ float2 s_c[JAC_CH];           // phix / vz^2, phiy / vz^2
    __shared__ int4 s_e[JAC_CH];             // basis row offsets of b, c, a; Jacobian row offset
    const int N = ctl.N, K = m.K, KP = m.KP, V = m.V, KTP = m.KTP;
    const int tid = threadIdx.x;
    const float4 *geo = b.geo + (size_t)f * V;
    const float *Rg = b.R + f * 9, *dR = b.dR + f * 27;
    const float *tau = b.xe + (size_t)f * KTP + K;
    const float phix = b.cam[f * 4], phiy = b.cam[f * 4 + 1];
    const Fragment *frags = b.frag + (size_t)f * NMAX;
    const float *fg = b.fgrad + (size_t)f * 5 * NMAX;
    float *Jf = b.J + (size_t)f * NMAX * KTP;
    float R[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = Rg[i];
    const uint32_t mg = 0xFFFFFFFFu / (uint32_t)K + 1u;   // i / K = umulhi(i, mg) for i < 2^16
    for (int c0 = blockIdx.x * JAC_CH; c0 < N; c0 += gridDim.x * JAC_CH) {
        const int cnt = min(JAC_CH, N - c0);
        if (tid < cnt) {
            const int n = c0 + tid;
            const Fragment fr = frags[n];
            const int4 tc = __ldg(m.tl4 + fr.tri);
            const int ib = tc.x, ic = tc.y, ia = tc.z;
            const float al = fr.al, be = fr.be, ga = (1 - fr.al) - fr.be;
            const float4 gb = geo[ib], gc = geo[ic], ga4 = geo[ia];
            const float px = (gb.x * al + gc.x * be) + ga4.x * ga;
            const float py = (gb.y * al + gc.y * be) + ga4.y * ga;
            const float pz = (gb.z * al + gc.z * be) + ga4.z * ga;
            float bX, bY, bZ, cX, cY, cZ, aX, aY, aZ;
            camera_coords(R, tau, gb.x, gb.y, gb.z, bX, bY, bZ);
            camera_coords(R, tau, gc.x, gc.y, gc.z, cX, cY, cZ);
            camera_coords(R, tau, ga4.x, ga4.y, ga4.z, aX, aY, aZ);
            const float vx = (bX * al + cX * be) + aX * ga;
            const float vy = (bY * al + cY * be) + aY * ga;
            const float vz = (bZ * al + cZ * be) + aZ * ga;
            const float ivz = 1.0f / vz, ivz2 = ivz * ivz;
            const float gx = fg[n], gy = fg[NMAX + n];
            s_w[tid] = make_float4(al, be, ga, gx);
            s_v[tid] = make_float4(vx, vy, vz, gy);
            s_c[tid] = make_float2(phix * ivz2, phiy * ivz2);
            s_e[tid] = make_int4(ib * 3 * KP, ic * 3 * KP, ia * 3 * KP, n * KTP);
            float *row = Jf + (size_t)n * KTP;
            row[K + 0] = -(gx * (phix * ivz) + gy * 0.0f);
            row[K + 1] = -(gx * 0.0f + gy * (phiy * ivz));
            row[K + 2] = -(gx * (((-phix) * vx) * ivz2) + gy * (((-phiy) * vy) * ivz2));
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float *d = dR + 9 * j;
                const float dvx = (d[0] * px + d[3] * py) + d[6] * pz;
                const float dvy = (d[1] * px + d[4] * py) + d[7] * pz;
                const float dvz = (d[2] * px + d[5] * py) + d[8] * pz;
                const float dWx = (phix * ivz2) * (vz * dvx - vx * dvz);
                const float dWy = (phiy * ivz2) * (vz * dvy - vy * dvz);
                row[K + 3 + j] = -(gx * dWx + gy * dWy);
            }
            for (int j = m.KT; j < KTP; ++j) row[j] = 0.0f;
        }
        __syncthreads();
#pragma unroll 2
        for (int i = tid; i < cnt * K; i += JAC_THREADS) {
            const int nl = (int)__umulhi((uint32_t)i, mg), k = i - nl * K;
            const float4 w = s_w[nl], v = s_v[nl];
            const float2 cc = s_c[nl];
            const int4 e = s_e[nl];
            const float *eb = m.E + e.x + k, *ec = m.E + e.y + k, *ea = m.E + e.z + k;
            const float tx = (__ldg(eb) * w.x + __ldg(ec) * w.y) + __ldg(ea) * w.z;
            const float ty = (__ldg(eb + KP) * w.x + __ldg(ec + KP) * w.y) + __ldg(ea + KP) * w.z;
            const float tz = (__ldg(eb + 2 * KP) * w.x + __ldg(ec + 2 * KP) * w.y) + __ldg(ea + 2 * KP) * w.z;
            const float REX = (tx * R[0] + ty * R[3]) + tz * R[6];
            const float REY = (tx * R[1] + ty * R[4]) + tz * R[7];
            const float REZ = (tx * R[2] + ty * R[5]) + tz * R[8];
            const float nwx = cc.x * (REX * v.z - REZ * v.x);
            const float nwy = cc.y * (REY * v.z - REZ * v.y);
            Jf[e.w + k] = -(w.w * nwx + v.w * nwy);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------
// Normal equations of the image term (derivative_computer.cu:135-164): rows of
// d(gx/|g|)/dtheta and d(gy/|g|)/dtheta, H = tau * sum(row row^T), g = -tau * sum(w row).
// The reference sums with cublasSgemm in the library's order; the order here is fixed and
// shared with the oracle: fragments in chunks of NE_CH, each chunk summed from zero with one
// FP64 fused multiply-add per row and entry in fragment order (x row, then y row), the chunk
// sums then added in chunk order. The rows are floats, so every product is exact in FP64.
// k_normal_eq writes one partial per chunk (NE_BPF blocks per frame, each looping over
// chunks); rows are staged 32 fragments at a time in shared memory as doubles and every
// thread owns a 4x4 block of the upper triangle. k_normal_eq_reduce adds the chunk partials.

constexpr int NE_THREADS = 256;
constexpr int NE_CH = 256;                   // fragments per chunk (the unit of the sum order)
constexpr int NE_SUB = 32;                   // fragments staged in shared memory at a time
constexpr int NE_BPF = 32;                   // blocks per frame
constexpr int NE_MAXCH = NMAX / NE_CH;       // chunk partials per frame at most
static_assert(NE_THREADS == NE_CH && NE_SUB == 32 && NE_THREADS == 8 * 32, "thread mapping of the row build");

// Chunk partials are sized for the widest layout the normal-equation kernels have used:
// 132 tiles of 4 x 8 doubles plus a row (KTP <= 88); the 8 x 8 tensor-core tiles need less.
constexpr int NE_TILES = 132;

__host__ __device__ __forceinline__ int ne_part_stride(int KTP)
{
    return NE_TILES * 32 + KTP;   // the widest partial layout of the normal-equation kernels
}

// Rows of one chunk of NE_CH fragments: per-fragment scalars and neighbour indices are
// staged once per chunk (one thread per fragment); a thread then builds fragment
// 4*warp + lane/8 of each 32-fragment stage at columns 8*g + lane%8, its four neighbour
// rows of J loaded one stage ahead.
constexpr int NE_GRP = 11;                   // column groups of 8: KTP <= 88 (K <= 82)

struct ChunkHead {
    int nb[4][NE_CH];
    float pre[NE_CH], dx[NE_CH], dy[NE_CH];
    double w[2 * NE_CH];
};

__device__ __forceinline__ void chunk_head(ChunkHead &hd, const float *fg, const int32_t *nb, int c0, int cnt)
{
    const int q = threadIdx.x, n = c0 + q;
    float pre = 0.0f, dx = 0.0f, dy = 0.0f, wx = 0.0f, wy = 0.0f;
    int k0 = 0, k1 = 0, k2 = 0, k3 = 0;
    if (q < cnt) {
        const float gx = fg[n], gy = fg[NMAX + n], h = fg[2 * NMAX + n];
        pre = (float)(1.0 / (0.001 + (double)(h * h * h)));
        dx = 2 * gx;
        dy = 2 * gy;
        wx = fg[3 * NMAX + n];
        wy = fg[4 * NMAX + n];
        k0 = nb[n]; k1 = nb[NMAX + n]; k2 = nb[2 * NMAX + n]; k3 = nb[3 * NMAX + n];
    }
    hd.pre[q] = pre; hd.dx[q] = dx; hd.dy[q] = dy;
    hd.nb[0][q] = k0; hd.nb[1][q] = k1; hd.nb[2][q] = k2; hd.nb[3][q] = k3;
    hd.w[2 * q] = (double)wx;
    hd.w[2 * q + 1] = (double)wy;
}

template <int GRP>
__device__ __forceinline__ void chunk_prefetch(float (&v)[GRP][4], const ChunkHead &hd, const float *Jf,
                                               int KT, int KTP, int q, int cnt, int a_low)
{
    const bool live = q < cnt;
    const int r0 = hd.nb[0][q], r1 = hd.nb[1][q], r2 = hd.nb[2][q], r3 = hd.nb[3][q];
#pragma unroll
    for (int g = 0; g < GRP; ++g) {
        const int a = 8 * g + a_low;
        const bool use = live && a < KT;
        v[g][0] = use ? Jf[(size_t)r0 * KTP + a] : 0.0f;
        v[g][1] = use ? Jf[(size_t)r1 * KTP + a] : 0.0f;
        v[g][2] = use ? Jf[(size_t)r2 * KTP + a] : 0.0f;
        v[g][3] = use ? Jf[(size_t)r3 * KTP + a] : 0.0f;
    }
}

// Chain rule through the normalised gradient (newfuncs.cu:417-463) at one column.
__device__ __forceinline__ void chain_value(const float (&vv)[4], float pre, float diffx, float diffy,
                                            float &ox, float &oy)
{
    const float dh = vv[1] - vv[0];
    const float dv = vv[3] - vv[2];
    const float X = (-diffy) * (-dh) - (-diffx) * (-dv);
    ox = ((-pre) * (-diffy)) * X;
    oy = (pre * (-diffx)) * X;
}

// FP64 tensor-core form of the exact sum: mma.sync m8n8k4 f64 updates an 8x8 tile with four
// rows k = 0..3 as the fused multiply-add chain d = fma(a3, b3, fma(a2, b2, fma(a1, b1,
// fma(a0, b0, c)))) (checked on B200 against CPU emulation: no mismatch in 4.2M entries; the
// parity tests check H and g bit for bit). Four rows are two fragments' x and y rows in
// order, so the chain is exactly the oracle's. Tiles of 8x8 cover the upper triangle of a
// P8 x P8 matrix whose column KT holds the weights w (so the column KT of the sum is g).
constexpr int NE_P8 = 88;                    // padded width: parameters + weight column, <= 88
constexpr int NE_T8 = NE_P8 / 8;             // 11 tile rows / columns
constexpr int NE_NT8 = NE_T8 * (NE_T8 + 1) / 2;   // 66 tiles
constexpr int NE_TPW = (NE_NT8 + 7) / 8;     // tiles per warp (8 warps)

__device__ __forceinline__ void ne_tile8(int t, int &bi, int &bj)
{
    bi = 0;
    while (t >= NE_T8 - bi) { t -= NE_T8 - bi; ++bi; }
    bj = bi + t;
}

__host__ __device__ __forceinline__ int ne_part_stride8() { return NE_NT8 * 64; }

__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// Rows are staged in shared memory as doubles (converted once when built), row pitch NE_PD:
// 92 doubles puts the four rows a warp reads at once on disjoint bank groups.
constexpr int NE_PD = NE_P8 + 4;

// Tile list in ne_tile8's order, as a compile-time table.
struct NeTiles {
    int bi[NE_NT8], bj[NE_NT8];
};
__host__ __device__ constexpr NeTiles make_ne_tiles()
{
    NeTiles t{};
    int k = 0;
    for (int i = 0; i < NE_T8; ++i)
        for (int j = i; j < NE_T8; ++j) { t.bi[k] = i; t.bj[k] = j; ++k; }
    return t;
}

// The tensor-core updates of warp W (tiles W, W + 8, ...) over the fragment pairs of one
// stage: a lane loads its row's value in each of the 11 column blocks once per pair and
// feeds every tile from those registers.
template <int W>
__device__ __forceinline__ void ne_pairs(double (&acc)[NE_TPW][2], const double *rows, int cn, int kr, int fr8)
{
    constexpr NeTiles TT = make_ne_tiles();
    constexpr int NT = (NE_NT8 - W + 7) / 8;
    for (int q = 0; q + 2 <= cn; q += 2) {
        const double *rk = rows + (size_t)(2 * q + kr) * NE_PD + fr8;
        double v[NE_T8];
#pragma unroll
        for (int c = 0; c < NE_T8; ++c) v[c] = rk[8 * c];
#pragma unroll
        for (int j = 0; j < NT; ++j) dmma_884(acc[j][0], acc[j][1], v[TT.bi[W + 8 * j]], v[TT.bj[W + 8 * j]]);
    }
}


__global__ void __launch_bounds__(NE_THREADS, 2) k_normal_eq(DModel m, DBatch b)
{
    if ((int)blockIdx.y >= active_n(b)) return;
    const int f = b.act[blockIdx.y];
    const FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) prof_count(b, KID_NORMAL_EQ);
    extern __shared__ __align__(16) double nesd[];  // rows [2][2*NE_SUB][NE_PD]
    const int KTP = m.KTP, KT = m.KT;
    __shared__ ChunkHead hd;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int a_low = lane & 7, q_me = 4 * warp + (lane >> 3);
    const int N = ctl.N;
    const int nch = (N + NE_CH - 1) / NE_CH;
    const float *Jf = b.J + (size_t)f * NMAX * KTP;
    const int32_t *nb = b.nb + (size_t)f * 4 * NMAX;
    const float *fg = b.fgrad + (size_t)f * 5 * NMAX;
    const int stride = ne_part_stride8();
    // this warp's tiles: t = warp + 8 * j
    int tbi[NE_TPW], tbj[NE_TPW];
#pragma unroll
    for (int j = 0; j < NE_TPW; ++j) {
        const int t = warp + 8 * j;
        if (t < NE_NT8) ne_tile8(t, tbi[j], tbj[j]); else { tbi[j] = -1; tbj[j] = -1; }
    }
    const int kr = lane & 3, fr8 = lane >> 2;        // fragment row k and tile row/column
    for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        double acc[NE_TPW][2];
#pragma unroll
        for (int j = 0; j < NE_TPW; ++j) acc[j][0] = acc[j][1] = 0.0;
        const int c0 = ch * NE_CH, cnt = min(N, c0 + NE_CH) - c0;
        const int nsub = (cnt + NE_SUB - 1) / NE_SUB;
        __syncthreads();                          // the previous chunk is done with hd and the rows
        chunk_head(hd, fg, nb, c0, cnt);
        __syncthreads();
        for (int it = 0; it < nsub; ++it) {
            double *rows = nesd + (size_t)(it & 1) * 2 * NE_SUB * NE_PD;
            {
                float v[NE_GRP][4];
                const int ql = q_me, q = it * NE_SUB + ql;
                chunk_prefetch<NE_GRP>(v, hd, Jf, KT, KTP, q, cnt, a_low);
                const float pre = hd.pre[q], diffx = hd.dx[q], diffy = hd.dy[q];
                const bool live = q < cnt;
#pragma unroll
                for (int g = 0; g < NE_GRP; ++g) {
                    const int a = 8 * g + a_low;
                    if (a >= NE_P8) continue;
                    float ox = 0.0f, oy = 0.0f;
                    if (live) {
                        if (a < KT) chain_value(v[g], pre, diffx, diffy, ox, oy);
                        else if (a == KT) { ox = (float)hd.w[2 * q]; oy = (float)hd.w[2 * q + 1]; }
                    }
                    rows[(2 * ql) * NE_PD + a] = (double)ox;
                    rows[(2 * ql + 1) * NE_PD + a] = (double)oy;
                }
            }
            __syncthreads();
            const int cn = min(NE_SUB, cnt - it * NE_SUB);
            // pairs of fragments on the tensor cores
            switch (warp) {
            case 0: ne_pairs<0>(acc, rows, cn, kr, fr8); break;
            case 1: ne_pairs<1>(acc, rows, cn, kr, fr8); break;
            case 2: ne_pairs<2>(acc, rows, cn, kr, fr8); break;
            case 3: ne_pairs<3>(acc, rows, cn, kr, fr8); break;
            case 4: ne_pairs<4>(acc, rows, cn, kr, fr8); break;
            case 5: ne_pairs<5>(acc, rows, cn, kr, fr8); break;
            case 6: ne_pairs<6>(acc, rows, cn, kr, fr8); break;
            default: ne_pairs<7>(acc, rows, cn, kr, fr8); break;
            }
            // an odd last fragment: this thread's two entries of each tile, same chain
            if (cn & 1) {
                const int q = cn - 1;
                const double *rx = rows + (size_t)(2 * q) * NE_PD, *ry = rx + NE_PD;
#pragma unroll
                for (int j = 0; j < NE_TPW; ++j) {
                    if (tbi[j] < 0) continue;
                    const int r = 8 * tbi[j] + fr8, c = 8 * tbj[j] + 2 * kr;
#pragma unroll
                    for (int i = 0; i < 2; ++i)
                        acc[j][i] = fma(ry[r], ry[c + i], fma(rx[r], rx[c + i], acc[j][i]));
                }
            }
        }
        double *part = b.ne_part + ((size_t)f * NE_MAXCH + ch) * stride;
#pragma unroll
        for (int j = 0; j < NE_TPW; ++j) {
            if (tbi[j] < 0) continue;
            const int t = warp + 8 * j;
            *reinterpret_cast<double2 *>(part + t * 64 + fr8 * 8 + 2 * kr) = make_double2(acc[j][0], acc[j][1]);
        }
    }
}

// Sum of the chunk partials in chunk order: H = tau*S, g = -tau*(column KT of S).
__global__ void __launch_bounds__(NE_THREADS) k_normal_eq_reduce(DModel m, DBatch b)
{
    if ((int)blockIdx.y >= active_n(b)) return;
    const int f = b.act[blockIdx.y];
    const FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    const int KTP = m.KTP, KT = m.KT;
    const int stride = ne_part_stride8();
    const int nch = (ctl.N + NE_CH - 1) / NE_CH;
    const double *part = b.ne_part + (size_t)f * NE_MAXCH * stride;
    const double tau = 25.0;
    float *H = b.H + (size_t)f * KTP * KTP;
    // one entry per thread: tile t, position p; the chunk values are loaded eight at a time
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NE_NT8 * 64; e += gridDim.x * blockDim.x) {
        const int t = e >> 6, pos = e & 63;
        int bi, bj;
        ne_tile8(t, bi, bj);
        const int a = 8 * bi + (pos >> 3), c = 8 * bj + (pos & 7);
        if (a > c || c > KT || a >= KT) continue;
        const double *p = part + e;
        double s = 0.0;
        int q = 0;
        for (; q + 8 <= nch; q += 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = p[(size_t)(q + u) * stride];
#pragma unroll
            for (int u = 0; u < 8; ++u) s += v[u];
        }
        for (; q < nch; ++q) s += p[(size_t)q * stride];
        if (c < KT) {
            const float v = (float)(tau * s);
            H[(size_t)a * KTP + c] = v;
            H[(size_t)c * KTP + a] = v;
        } else {
            b.g[(size_t)f * KTP + a] = (float)(-tau * s);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Log-barrier gradient and Gauss-Newton Hessian (logbarrier_initializer.cu:1272-1843) added
// to the image system, one block per frame.

// The barrier Hessian's tensor-core updates of warp W over the 4 x 51 constraint rows (FP32
// in shared memory, pitch NE_P8), four consecutive rows per step.
template <int W>
__device__ __forceinline__ void bar_hessian(double (&acc)[NE_TPW][2], const float *Fm, int KTP, int kr, int fr8)
{
    constexpr NeTiles TT = make_ne_tiles();
    constexpr int NT = (NE_NT8 - W + 7) / 8;
    for (int t = 0; t < 4 * NL; t += 4) {
        const float *rk = Fm + (size_t)(t + kr) * KTP + fr8;
        double v[NE_T8];
#pragma unroll
        for (int c = 0; c < NE_T8; ++c) v[c] = (double)rk[8 * c];
#pragma unroll
        for (int j = 0; j < NT; ++j) dmma_884(acc[j][0], acc[j][1], v[TT.bi[W + 8 * j]], v[TT.bj[W + 8 * j]]);
    }
}

__global__ void __launch_bounds__(256) k_barrier_full(DModel m, DBatch b, int ft_bounds)
{
    if ((int)blockIdx.x >= active_n(b)) return;
    const int f = b.act[blockIdx.x];
    const FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    if (threadIdx.x == 0) prof_count(b, KID_BARRIER);
    extern __shared__ float bsm[];
    const int KT = m.KT, KTP = m.KTP, K = m.K;
    float *Fm = bsm;                              // [4*NL][NE_P8], zeros right of KT
    __shared__ float G[4][NL];
    __shared__ float s_p[NL][3];
    __shared__ float s_v[NL][3], s_ivz[NL], s_ivz2[NL];
    __shared__ int s_lis[NL];
    __shared__ float s_R[9], s_dR[27];
    const int tid = threadIdx.x;
    const float *x = b.x + (size_t)f * KTP;       // the accepted point (= evaluation point)
    const float *R = b.R + f * 9, *dR = b.dR + f * 27;
    const float *tau = x + K;
    const float4 *geo = b.geo + (size_t)f * m.V;
    const float *cam = b.cam + f * 4;
    const float phix = cam[0], phiy = cam[1], cx = cam[2], cy = cam[3];
    const float fs = b.face_size[f];
    const float *bnd = b.bounds + (size_t)f * 4 * NL;
    const float *xl = b.xl + f * NL, *yl = b.yl + f * NL;
    if (tid >= 64 && tid < 64 + 36) {
        const int q = tid - 64;
        if (q < 9) s_R[q] = R[q]; else s_dR[q - 9] = dR[q - 9];
    }
    if (tid < NL) {
        const int v = m.lis[tid];
        s_lis[tid] = v;
        const float4 pv = geo[v];
        const float p0 = pv.x, p1 = pv.y, p2 = pv.z;
        s_p[tid][0] = p0; s_p[tid][1] = p1; s_p[tid][2] = p2;
        const float r1p = (R[0] * p0 + R[3] * p1) + R[6] * p2;
        const float r2p = (R[1] * p0 + R[4] * p1) + R[7] * p2;
        const float r3p = (R[2] * p0 + R[5] * p1) + R[8] * p2;
        const float xproj = phix * ((r1p + tau[0]) / (r3p + tau[2])) + cx;
        const float yproj = phiy * ((r2p + tau[1]) / (r3p + tau[2])) + cy;
        G[0][tid] = 0.0f - ((xl[tid] + bnd[0 * NL + tid] * fs) - xproj);
        G[1][tid] = 0.0f - ((yl[tid] + bnd[1 * NL + tid] * fs) - yproj);
        G[2][tid] = 0.0f - ((xproj - bnd[2 * NL + tid] * fs) - xl[tid]);
        G[3][tid] = 0.0f - ((yproj - bnd[3 * NL + tid] * fs) - yl[tid]);
        // camera point of the landmark and its inverse depth, once per landmark
        const float vx = r1p + tau[0], vy = r2p + tau[1], vz = r3p + tau[2];
        s_v[tid][0] = vx; s_v[tid][1] = vy; s_v[tid][2] = vz;
        const float ivz = 1.0f / vz;
        s_ivz[tid] = ivz;
        s_ivz2[tid] = ivz * ivz;
    }
    __syncthreads();
    // rows of the constraint gradients: warps take landmarks (i = warp + 8 q), lanes take
    // columns (a = lane + 32 c). Per column the basis values of all the warp's landmarks are
    // loaded before any is used, so that their loads are in flight together; the rotation and
    // its derivatives come from shared memory.
    constexpr int BQ = (NL + 7) / 8;
    const int warp = tid >> 5;
    for (int a = tid & 31; a < NE_P8; a += 32) {
        float eb[BQ][3];
#pragma unroll
        for (int q = 0; q < BQ; ++q) {
            const int i = warp + 8 * q;
            eb[q][0] = eb[q][1] = eb[q][2] = 0.0f;
            if (i < NL && a < K) {
                const float *ex = m.E + (size_t)s_lis[i] * 3 * m.KP;
                eb[q][0] = __ldg(ex + a);
                eb[q][1] = __ldg(ex + m.KP + a);
                eb[q][2] = __ldg(ex + 2 * m.KP + a);
            }
        }
#pragma unroll
        for (int q = 0; q < BQ; ++q) {
            const int i = warp + 8 * q;
            if (i >= NL) continue;
            const float p0 = s_p[i][0], p1 = s_p[i][1], p2 = s_p[i][2];
            const float vx = s_v[i][0], vy = s_v[i][1], vz = s_v[i][2];
            const float ivz = s_ivz[i], ivz2 = s_ivz2[i];
            float wx = 0.0f, wy = 0.0f;
            if (a < K) {
                const float RIX = eb[q][0], RIY = eb[q][1], RIZ = eb[q][2];
                const float dvx = (RIX * s_R[0] + RIY * s_R[3]) + RIZ * s_R[6];
                const float dvy = (RIX * s_R[1] + RIY * s_R[4]) + RIZ * s_R[7];
                const float dvz = (RIX * s_R[2] + RIY * s_R[5]) + RIZ * s_R[8];
                wx = (phix * ivz2) * (dvx * vz - dvz * vx);
                wy = (phiy * ivz2) * (dvy * vz - dvz * vy);
            } else if (a < KT) {
                const int cidx = a - K;
                if (cidx == 0) { wx = phix * ivz; wy = 0.0f; }
                else if (cidx == 1) { wx = 0.0f; wy = phiy * ivz; }
                else if (cidx == 2) { wx = ((-phix) * vx) * ivz2; wy = ((-phiy) * vy) * ivz2; }
                else {
                    const float *d = s_dR + 9 * (cidx - 3);
                    const float dvx = (d[0] * p0 + d[3] * p1) + d[6] * p2;
                    const float dvy = (d[1] * p0 + d[4] * p1) + d[7] * p2;
                    const float dvz = (d[2] * p0 + d[5] * p1) + d[8] * p2;
                    wx = (phix * ivz2) * (vz * dvx - vx * dvz);
                    wy = (phiy * ivz2) * (vz * dvy - vy * dvz);
                }
            }
            const bool live = a < KT;
            Fm[(0 * NL + i) * NE_P8 + a] = live ? -wx / G[0][i] : 0.0f;
            Fm[(1 * NL + i) * NE_P8 + a] = live ? -wy / G[1][i] : 0.0f;
            Fm[(2 * NL + i) * NE_P8 + a] = live ? wx / G[2][i] : 0.0f;
            Fm[(3 * NL + i) * NE_P8 + a] = live ? wy / G[3][i] : 0.0f;
        }
    }
    __syncthreads();
    const float *lb = m.eps_b + (ft_bounds ? 2 : 0) * K;
    const float *ub = m.eps_b + (ft_bounds ? 3 : 1) * K;
    float *H = b.H + (size_t)f * KTP * KTP;
    float *gv = b.g + (size_t)f * KTP;
    // gradient: column sums over landmarks, set by set (the oracle's order)
    if (tid < KT) {
        const int a = tid;
        double gs = 0.0;
        for (int i = 0; i < NL; ++i)
            for (int s = 0; s < 4; ++s) gs += (double)Fm[(s * NL + i) * NE_P8 + a];
        float ga = (float)gs;
        if (a < K) {
            const float fub = x[a] - ub[a];
            const float flb = lb[a] - x[a];
            ga = ga + (-1.0f / fub + 1.0f / flb);
        }
        gv[a] += ga;
    }
    // Hessian: H = sum over the 204 constraint rows (set, then landmark) of F_t^T F_t, each entry
    // one FP64 fused multiply-add chain in row order, the oracle's order (the terms are
    // products of floats, exact in FP64). On the FP64 tensor cores: mma.sync m8n8k4 adds four
    // consecutive rows to an 8x8 tile as fma(a3, b3, fma(a2, b2, fma(a1, b1, fma(a0, b0, c)))),
    // the same chain; 66 tiles of the upper triangle, warp W taking tiles W, W + 8, ...
    {
        const int lane = tid & 31, warp = tid >> 5;
        const int kr = lane & 3, fr8 = lane >> 2;
        double acc[NE_TPW][2];
#pragma unroll
        for (int j = 0; j < NE_TPW; ++j) acc[j][0] = acc[j][1] = 0.0;
        switch (warp) {
        case 0: bar_hessian<0>(acc, Fm, NE_P8, kr, fr8); break;
        case 1: bar_hessian<1>(acc, Fm, NE_P8, kr, fr8); break;
        case 2: bar_hessian<2>(acc, Fm, NE_P8, kr, fr8); break;
        case 3: bar_hessian<3>(acc, Fm, NE_P8, kr, fr8); break;
        case 4: bar_hessian<4>(acc, Fm, NE_P8, kr, fr8); break;
        case 5: bar_hessian<5>(acc, Fm, NE_P8, kr, fr8); break;
        case 6: bar_hessian<6>(acc, Fm, NE_P8, kr, fr8); break;
        default: bar_hessian<7>(acc, Fm, NE_P8, kr, fr8); break;
        }
#pragma unroll
        for (int j = 0; j < NE_TPW; ++j) {
            const int t = warp + 8 * j;
            if (t >= NE_NT8) continue;
            int bi, bj;
            ne_tile8(t, bi, bj);
            const int a = 8 * bi + fr8;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int c = 8 * bj + 2 * kr + i;
                if (a > c || c >= KT) continue;
                float hv = (float)acc[j][i];
                if (a == c && a < K) {
                    const float fub = x[a] - ub[a];
                    const float flb = lb[a] - x[a];
                    const float nu = (float)(-1.0 / ((double)fub + 1e-12));
                    const float nl = (float)(1.0 / ((double)flb + 1e-12));
                    hv = hv + (nu * nu + nl * nl);
                }
                H[(size_t)c * KTP + a] += hv;
                if (a != c) H[(size_t)a * KTP + c] += hv;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// FP64 Cholesky solve (solver.h:70-105, cuSOLVER DPOTRF/DPOTRS in the reference) of the shape
// system, one block per frame, then the first trial of the line search.
//
// Arithmetic (shared with the oracle's solve_shape): pivots l_jj = sqrt(s_j) with reciprocal
// r_j = 1 / l_jj; L(i,j) = t_ij * r_j, where t_ij is a_ij minus L(i,k) L(j,k) for k = 0, 1, ...
// in increasing k (each product and difference rounded); forward y_i = (g_i - sum_k L(i,k) y_k)
// * r_i with terms in increasing k; back x_i = (y_i - sum_k L(k,i) x_k) * r_i with terms in
// decreasing k. (cuSOLVER's order is the library's; the reciprocal is one rounding per column.)
//
// The lower triangle is held in registers: thread (tr, tc) = (tid % 16, tid / 16) owns the
// entries (i, l) with i = tr + 16a, l = tc + 16b, i >= l. Step j: every thread reads column j
// as its owners left it in shared memory (pivot included) and r_j as the pivot's owner formed
// it, forms the scaled entries it needs, and subtracts L(i,j) L(l,j) from its entries right of
// column j: the register block holding column j + 1 first, after which the owners of column
// j + 1 store it and the owner of its pivot forms l and r for the next step while the other
// blocks are updated. Each entry so receives its updates in increasing j, the sequence of the
// oracle's left-looking dot products. One barrier per step; the two substitutions run in one
// warp, four rows per lane, the newly known value broadcast by shuffle.
//
// The steps run in groups of 16 columns, one group per register block, each group its own
// instantiation. Every register block is then named by a compile-time index, and the finished
// blocks are skipped without tests. Selecting the next column's block at run time instead moved
// the whole block array into local memory (a 288-byte stack frame). Keeping it in registers
// while updating every block under run-time tests measured slower still: 1.59 µs per
// evaluation, against 1.10 µs with the stack and 0.96 µs in groups. The substitutions with the
// reciprocals in registers and no stores inside the passes took it to 0.90 µs, and the pivot
// formed one step ahead by its owner to 0.86 µs.

constexpr int SV_THREADS = 256;
constexpr int SV_MAXN = 128;

__host__ __device__ __forceinline__ size_t solve_smem(int n)
{
    return ((size_t)n * n + 4 * SV_MAXN + 2) * sizeof(double);
}

// One substitution pass of the warp: rows i = lane + 32 q (q < 4) start from t[q]; for each
// step k (ascending when FWD, descending otherwise) the owner of row k (lane k % 32) forms
// x_k = t_k r_k from its own registers and broadcasts it, and every row i after k in that
// order subtracts coef(i, k) x_k. The steps run in four segments of 32 with the row slot q a
// compile-time index, and nothing is stored inside the pass, so that the coefficient loads of
// later steps can be issued early. x of the lane's own rows ends in xm[].
template <bool FWD>
__device__ __forceinline__ void sv_substitute(int n, double (&t)[4], const double (&rm)[4], double (&xm)[4],
                                              const double *Lf)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int q = FWD ? s : 3 - s;
        if (32 * q >= n) continue;
#pragma unroll 4
        for (int u = 0; u < 32; ++u) {
            const int kk = FWD ? u : 31 - u;
            const int k = 32 * q + kk;
            if (k >= n) { if (FWD) break; else continue; }
            const double xo = t[q] * rm[q];             // meaningful in the owner lane
            if (lane == kk) xm[q] = xo;
            const double xk = __shfl_sync(0xffffffffu, xo, kk);
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                if (FWD ? qq < q : qq > q) continue;
                const int i = lane + 32 * qq;
                // forward: L(i,k) for i > k (column k); back: L(k,i) for i < k (column i)
                if (FWD ? (i > k && i < n) : (i < k)) t[qq] -= (FWD ? Lf[(size_t)k * n + i] : Lf[(size_t)i * n + k]) * xk;
            }
        }
    }
}

// The trailing update of step j (column j scaled into ci, cl), with column j + 1 in register
// block B: the blocks (a, B) first; then the owners of column j + 1 store it, and the owner of
// its pivot forms l = sqrt(s) and r = 1 / l (both correctly rounded) for the next step while
// the other blocks (a, bb > B) are updated. Blocks left of B receive no more updates.
template <int RB, int B>
__device__ __forceinline__ void sv_update(double (&v)[RB][RB], const double (&ci)[RB], const double (&cl)[RB],
                                          int tr, int tc, int j, int n, double *rn, double *Lf, double *rv)
{
#pragma unroll
    for (int a = B; a < RB; ++a) {
        const int i = tr + 16 * a, l = tc + 16 * B;
        if (l > j && i >= l && i < n) v[a][B] -= ci[a] * cl[B];
    }
    const int jn = j + 1;
    if (jn < n && tc == (jn & 15)) {
#pragma unroll
        for (int a = B; a < RB; ++a) {
            const int i = tr + 16 * a;
            if (i >= jn && i < n) rn[i] = v[a][B];
        }
        if (tr == (jn & 15)) {
            const double sn = v[B][B];
            if (sn > 0.0) {
                const double ln = sqrt(sn);
                Lf[(size_t)jn * n + jn] = ln;
                rv[jn] = __drcp_rn(ln);
            }
        }
    }
#pragma unroll
    for (int a = B + 1; a < RB; ++a)
#pragma unroll
        for (int bb = B + 1; bb <= a; ++bb) {
            const int i = tr + 16 * a, l = tc + 16 * bb;
            if (l > j && i >= l && i < n) v[a][bb] -= ci[a] * cl[bb];
        }
}

// Steps j of column group J (columns 16 J .. 16 J + 15), then the next group; false when a
// pivot is not positive (every thread reads the same pivot, so all return together). Blocks
// left of group J (bb < J) and rows above it (a < J) are finished: their columns l < 16 J <= j
// receive no more updates, so they are skipped statically.
template <int RB, int J>
__device__ __forceinline__ bool sv_factor(double (&v)[RB][RB], double *raw, double *Lf, double *rv,
                                          int tr, int tc, int tid, int n)
{
    const int jend = min(n, 16 * J + 16);
    for (int j = 16 * J; j < jend; ++j) {
        const double *rj = raw + (j & 1) * SV_MAXN;
        const double sj = rj[j];
        if (!(sj > 0.0)) return false;
        const double r = rv[j];                          // formed by the pivot's owner in step j - 1
        if (tid > j && tid < n) Lf[(size_t)j * n + tid] = rj[tid] * r;
        double ci[RB], cl[RB];
#pragma unroll
        for (int a = J; a < RB; ++a) {
            const int i = tr + 16 * a, l = tc + 16 * a;
            ci[a] = (i > j && i < n) ? rj[i] * r : 0.0;
            cl[a] = (l > j && l < n) ? rj[l] * r : 0.0;
        }
        double *rn = raw + ((j + 1) & 1) * SV_MAXN;
        if (j < 16 * J + 15) sv_update<RB, J>(v, ci, cl, tr, tc, j, n, rn, Lf, rv);
        else sv_update<RB, (J + 1 < RB ? J + 1 : J)>(v, ci, cl, tr, tc, j, n, rn, Lf, rv);
        __syncthreads();
    }
    if constexpr (J + 1 < RB) return sv_factor<RB, J + 1>(v, raw, Lf, rv, tr, tc, tid, n);
    else return true;
}

template <int RB>
__device__ __forceinline__ void solve_frame(const DModel &m, const DBatch &b, const Cfg &c, int stage, int f,
                                            FrameCtl &ctl, double *sm)
{
    const int n = m.KT, KTP = m.KTP, K = m.K;
    const int tid = threadIdx.x, tr = tid & 15, tc = tid >> 4;
    double *Lf = sm;                     // [n][n] column-major: the factor, for the substitutions
    double *raw = Lf + (size_t)n * n;    // [2][SV_MAXN] column j before its scaling (by step parity)
    double *rv = raw + 2 * SV_MAXN;      // [SV_MAXN] reciprocal pivots
    double *yv = rv + SV_MAXN;           // [SV_MAXN] forward, then back results
    const float *H = b.H + (size_t)f * KTP * KTP;
    const float *gv = b.g + (size_t)f * KTP;
    double v[RB][RB];
    const double lam_d = (double)c.damping;      // damped solve: H + lambda I (0: undamped)
#pragma unroll
    for (int a = 0; a < RB; ++a)
#pragma unroll
        for (int bb = 0; bb < RB; ++bb) {
            const int i = tr + 16 * a, l = tc + 16 * bb;
            v[a][bb] = (i < n && l < n && i >= l) ? (double)H[(size_t)l * KTP + i] : 0.0;
            if (i == l && i < n) v[a][bb] += lam_d;
        }
    // column 0 before scaling, pivot included
#pragma unroll
    for (int a = 0; a < RB; ++a)
        if (tc == 0 && tr + 16 * a < n) raw[tr + 16 * a] = v[a][0];
    if (tid == 0 && v[0][0] > 0.0) {
        const double l0 = sqrt(v[0][0]);
        Lf[0] = l0;
        rv[0] = __drcp_rn(l0);
    }
    __syncthreads();
    // Columns in register-block groups J (columns 16 J .. 16 J + 15), one instantiation per
    // group, so that every register block is named by a compile-time index.
    if (!sv_factor<RB, 0>(v, raw, Lf, rv, tr, tc, tid, n)) {    // block-uniform: the same pivot everywhere
        float *d = b.d + (size_t)f * KTP;
        for (int i = tid; i < n; i += SV_THREADS) d[i] = __int_as_float(0x7fc00000);
        if (tid == 0) {
            ctl.flags |= FLAG_CHOL_FAILED | FLAG_NAN_DIRECTION;
            end_shape_stage(c, ctl, stage, ctl.outer);
        }
        return;
    }
    // forward and back substitution in one warp
    if (tid < 32) {
        double t[4], rm[4], xm[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = tid + 32 * q;
            t[q] = i < n ? (double)gv[i] : 0.0;
            rm[q] = i < n ? rv[i] : 0.0;
            xm[q] = 0.0;
        }
        sv_substitute<true>(n, t, rm, xm, Lf);
        // y_i = t_i r_i: the value the owner of row i broadcast at step i
#pragma unroll
        for (int q = 0; q < 4; ++q) t[q] = xm[q];
        sv_substitute<false>(n, t, rm, xm, Lf);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = tid + 32 * q;
            if (i < n) yv[i] = xm[q];
        }
    }
    __syncthreads();
    const double y = tid < n ? yv[tid] : 0.0;
    // direction, its slope and the first trial point
    float *d = b.d + (size_t)f * KTP;
    float *dsm = reinterpret_cast<float *>(raw);
    if (tid < n) { const float dv = (float)(-y); d[tid] = dv; dsm[tid] = dv; }
    __syncthreads();
    if (isnan(dsm[0])) {
        if (tid == 0) {
            ctl.flags |= FLAG_NAN_DIRECTION;
            end_shape_stage(c, ctl, stage, ctl.outer);
        }
        return;
    }
    const int n_upd = stage == ST_FINETUNE ? K : n;
    const float t = 1.0f;
    const float *x = b.x + (size_t)f * KTP;
    float *xl = b.x_ls + (size_t)f * KTP;
    for (int a = tid; a < n_upd; a += SV_THREADS) xl[a] = x[a] + t * dsm[a];
    if (tid == 0) {
        double dg = 0.0;
        for (int a = 0; a < n; ++a) dg += (double)dsm[a] * (double)gv[a];
        ctl.l2base = (float)dg;
        ctl.mode = M_TRIAL;
        ctl.t = t;
        const int maxit = stage == ST_RIGID ? c.max_iters_rigid : c.max_iters_finetune;
        // the trial's tau_z (left as it was when the stage does not update the pose)
        const float tz = n_upd > K + 2 ? x[K + 2] + t * dsm[K + 2] : xl[K + 2];
        if (tz < 0.0f) {
            ctl.flags |= FLAG_STUCK_NEG_TZ;
            end_shape_stage(c, ctl, stage, maxit);
        }
    }
}

// RB = 6 register blocks for up to 96 unknowns, 8 up to 128: one kernel each, so that the
// smaller system is not held to the larger one's register count
template <int RB>
__global__ void __launch_bounds__(SV_THREADS) k_solve_t(DModel m, DBatch b, Cfg c, int stage)
{
    if ((int)blockIdx.x >= active_n(b)) return;
    const int f = b.act[blockIdx.x];
    FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    if (threadIdx.x == 0) prof_count(b, KID_SOLVE);
    extern __shared__ double ssm[];
    solve_frame<RB>(m, b, c, stage, f, ctl, ssm);
}

// ------------------------------------------------------------------------------------------
// Light system (derivative_computer.cu:235-312): dI/dlambda = L t (R n), chain rule, 3x3
// normal equations in FP64, Cholesky, first trial. One block per frame.

constexpr int LJ_U = 4;   // fragments per thread whose gathers are in flight together

__global__ void __launch_bounds__(256) k_lambda_jac(DModel m, DBatch b, Cfg c)
{
    if ((int)blockIdx.x >= active_n(b)) return;
    const int f = b.act[blockIdx.x];
    FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    __shared__ double s_red[8][12];
    __shared__ double s_L[9], s_y[3];
    __shared__ float s_g[3];
    const int tid = threadIdx.x, N = ctl.N;
    const float4 *geo = b.geo + (size_t)f * m.V;
    const float *R = b.R + f * 9;
    const float *tau = b.x + (size_t)f * m.KTP + m.K;
    const float *lam = b.lam + f * 4;
    const float Lint = b.Lint[f];
    const Fragment *frags = b.frag + (size_t)f * NMAX;
    float *Jl = b.J + (size_t)f * NMAX * m.KTP;   // rows of pitch 4
    // fragments LJ_U at a time, their gathers issued together (each thread still takes its
    // fragments in ascending order, so the FP64 sums below keep their order)
    for (int n0 = tid; n0 < N; n0 += 256 * LJ_U) {
        Fragment fr[LJ_U];
#pragma unroll
        for (int u = 0; u < LJ_U; ++u) {
            const int n = n0 + u * 256;
            fr[u] = n < N ? frags[n] : Fragment{0u, 0, 0.0f, 0.0f};
        }
        float rr[LJ_U][3];
#pragma unroll
        for (int u = 0; u < LJ_U; ++u) {
            float nn[3], t;
            if (ctl.shade_cached) {
                // the light fit's render of this geometry formed them (k_render)
                const int n = min(n0 + u * 256, N - 1);
                const float4 sn = b.shc[(size_t)f * NMAX + n];
                nn[0] = sn.x; nn[1] = sn.y; nn[2] = sn.z;
                t = b.sht[(size_t)f * NMAX + n];
            } else {
                const Shading sh = shade(m, geo, fr[u], R, tau, lam, Lint);
                nn[0] = sh.nn[0]; nn[1] = sh.nn[1]; nn[2] = sh.nn[2];
                t = sh.t;
            }
            const float Lt = Lint * t;
            const float r0 = Lt * nn[0], r1 = Lt * nn[1], r2 = Lt * nn[2];
#pragma unroll
            for (int j = 0; j < 3; ++j) rr[u][j] = (r0 * R[j] + r1 * R[j + 3]) + r2 * R[j + 6];
        }
#pragma unroll
        for (int u = 0; u < LJ_U; ++u) {
            const int n = n0 + u * 256;
            if (n >= N) break;
            *reinterpret_cast<float4 *>(Jl + (size_t)n * 4) = make_float4(rr[u][0], rr[u][1], rr[u][2], 0.0f);
        }
    }
    __syncthreads();
    const int32_t *nb = b.nb + (size_t)f * 4 * NMAX;
    const float *fg = b.fgrad + (size_t)f * 5 * NMAX;
    double acc[12];
    for (int q = 0; q < 12; ++q) acc[q] = 0.0;
    for (int n0 = tid; n0 < N; n0 += 256 * LJ_U) {
        float4 jr[LJ_U][4];
#pragma unroll
        for (int u = 0; u < LJ_U; ++u) {
            const int n = n0 + u * 256;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                jr[u][q] = n < N ? *reinterpret_cast<const float4 *>(Jl + (size_t)nb[q * NMAX + n] * 4) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
#pragma unroll
        for (int u = 0; u < LJ_U; ++u) {
            const int n = n0 + u * 256;
            if (n >= N) break;
            const float gx = fg[n], gy = fg[NMAX + n], h = fg[2 * NMAX + n];
            const float pre = (float)(1.0 / (0.001 + (double)(h * h * h)));
            float ox[3], oy[3];
            const float k0[3] = {jr[u][0].x, jr[u][0].y, jr[u][0].z}, k1[3] = {jr[u][1].x, jr[u][1].y, jr[u][1].z};
            const float k2[3] = {jr[u][2].x, jr[u][2].y, jr[u][2].z}, k3[3] = {jr[u][3].x, jr[u][3].y, jr[u][3].z};
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float vv[4] = {k0[j], k1[j], k2[j], k3[j]};
                chain_value(vv, pre, 2 * gx, 2 * gy, ox[j], oy[j]);
            }
            const double sx = fg[3 * NMAX + n], sy = fg[4 * NMAX + n];
            for (int a = 0; a < 3; ++a) {
                acc[9 + a] += sx * ox[a] + sy * oy[a];
                for (int bb = 0; bb < 3; ++bb) acc[a * 3 + bb] += (double)ox[a] * ox[bb] + (double)oy[a] * oy[bb];
            }
        }
    }
    for (int q = 0; q < 12; ++q)
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
    if ((tid & 31) == 0)
        for (int q = 0; q < 12; ++q) s_red[tid >> 5][q] = acc[q];
    __syncthreads();
    if (tid != 0) return;
    double tot[12];
    for (int q = 0; q < 12; ++q) { tot[q] = 0.0; for (int w = 0; w < 8; ++w) tot[q] += s_red[w][q]; }
    float Hf[9];
    for (int i = 0; i < 9; ++i) Hf[i] = (float)tot[i];
    for (int i = 0; i < 3; ++i) s_g[i] = (float)(-tot[9 + i]);
    // 3x3 Cholesky in the oracle's order (single thread)
    int ok = 1;
    for (int i = 0; i < 9; ++i) s_L[i] = (double)Hf[i];
    for (int j = 0; j < 3 && ok; ++j) {
        double s = s_L[j * 3 + j];
        for (int k = 0; k < j; ++k) s -= s_L[k * 3 + j] * s_L[k * 3 + j];
        if (!(s > 0.0)) { ok = 0; break; }
        const double ljj = sqrt(s);
        s_L[j * 3 + j] = ljj;
        for (int i = j + 1; i < 3; ++i) {
            double t = s_L[j * 3 + i];
            for (int k = 0; k < j; ++k) t -= s_L[k * 3 + i] * s_L[k * 3 + j];
            s_L[j * 3 + i] = t / ljj;
        }
    }
    float dl[3];
    if (ok) {
        for (int i = 0; i < 3; ++i) {
            double t = (double)s_g[i];
            for (int k = 0; k < i; ++k) t -= s_L[k * 3 + i] * s_y[k];
            s_y[i] = t / s_L[i * 3 + i];
        }
        for (int i = 2; i >= 0; --i) {
            double t = s_y[i];
            for (int k = i + 1; k < 3; ++k) t -= s_L[i * 3 + k] * s_y[k];
            s_y[i] = t / s_L[i * 3 + i];
        }
        for (int i = 0; i < 3; ++i) dl[i] = (float)(-s_y[i]);
    } else {
        for (int i = 0; i < 3; ++i) dl[i] = __int_as_float(0x7fc00000);
    }
    for (int j = 0; j < 3; ++j) { b.dlam[f * 4 + j] = dl[j]; b.glam[f * 4 + j] = s_g[j]; }
    const float l2 = (float)((double)dl[0] * s_g[0] + (double)dl[1] * s_g[1] + (double)dl[2] * s_g[2]);
    ctl.l2base = l2;
    ctl.mode = M_TRIAL;
    ctl.t = 1.0f;
    for (int j = 0; j < 3; ++j) b.lam_ls[f * 4 + j] = lam[j] + 1.0f * dl[j];
    // the first trial's -g.d test (model_fitter.cu:1044-1048) does not depend on the trial
    if ((double)(-l2) < 0.0003 || !(l2 == l2)) ctl.active = 0;
}

// Unblurred image and owner-triangle map of every rendering frame (renderer.cu:635-696).
__global__ void k_paint(DModel m, DBatch b, float *images, int32_t *tri_map)
{
    const int f = blockIdx.y;
    const FrameCtl &ctl = b.ctl[f];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < NPIX; p += gridDim.x * blockDim.x) {
        images[(size_t)f * NPIX + p] = 0.0f;
        tri_map[(size_t)f * NPIX + p] = -1;
    }
    if (!ctl.render) return;
    __syncthreads();
    // the clear above and the writes below touch disjoint work of one frame only when the
    // grid has a single block in x; the host launches it that way
    const float4 *geo = b.geo + (size_t)f * m.V;
    const float *R = b.R + f * 9;
    const float *tau = b.xe + (size_t)f * m.KTP + m.K;
    const float *lam = b.lam + f * 4;
    const Fragment *frags = b.frag + (size_t)f * NMAX;
    for (int n = threadIdx.x; n < ctl.N; n += blockDim.x) {
        const Fragment fr = frags[n];
        if (!(fr.pix_owner & 0x80000000u)) continue;
        const Shading s = shade(m, geo, fr, R, tau, lam, b.Lint[f]);
        const int p = fr.pix_owner & 0xFFFF;
        images[(size_t)f * NPIX + p] = s.tex;
        tri_map[(size_t)f * NPIX + p] = fr.tri;
    }
}

// Frames of the active list that render this round, in ascending order (one block).
__global__ void __launch_bounds__(1024) k_compact_render(DBatch b)
{
    __shared__ int s_warp[32];
    __shared__ int s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_base = 0;
    __syncthreads();
    const int na = active_n(b);
    for (int i0 = 0; i0 < na; i0 += 1024) {
        const int i = i0 + tid;
        const int f = i < na ? b.act[i] : -1;
        const int r = f >= 0 && b.ctl[f].render;
        const unsigned mask = __ballot_sync(0xffffffffu, r);
        if (lane == 0) s_warp[warp] = __popc(mask);
        __syncthreads();
        if (tid < 32) {
            int v = s_warp[tid], incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += t;
            }
            s_warp[tid] = incl - v;
        }
        __syncthreads();
        if (r) b.rlist[s_base + s_warp[warp] + __popc(mask & ((1u << lane) - 1u))] = f;
        __syncthreads();
        if (tid == 1023) s_base += s_warp[31] + __popc(mask);
        __syncthreads();
    }
    if (tid == 0) b.rcount[0] = s_base;
}

// Frames still running the current stage, in ascending order (one block, block-wide scan).
__global__ void __launch_bounds__(1024) k_compact_active(DBatch b, int *out)
{
    __shared__ int s_warp[32];
    __shared__ int s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_base = 0;
    __syncthreads();
    for (int f0 = 0; f0 < b.F; f0 += 1024) {
        const int f = f0 + tid;
        const int a = (f < b.F) ? b.ctl[f].active : 0;
        const unsigned mask = __ballot_sync(0xffffffffu, a);
        if (lane == 0) s_warp[warp] = __popc(mask);
        __syncthreads();
        if (tid < 32) {
            int v = s_warp[tid], incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += t;
            }
            s_warp[tid] = incl - v;
        }
        __syncthreads();
        if (a) b.act[s_base + s_warp[warp] + __popc(mask & ((1u << lane) - 1u))] = f;
        __syncthreads();
        if (tid == 1023) s_base += s_warp[31] + __popc(mask);
        __syncthreads();
    }
    if (tid == 0) {
        out[0] = s_base;
        out[1] = *b.err;
    }
}

// ------------------------------------------------------------------------------------------
// The subject's shape and albedo (renderer.cu:866-883,941-951): one thread per coordinate of a
// vertex (rows 0..3V-1: X, Y, Z planes) or albedo entry (rows 3V..4V-1); the basis row is a
// sequential fused multiply-add chain over k from 0, then added to the mean. In place on m, t.

__global__ void k_apply_identity(int V, int KA, int KB, float *m, const float *I, const float *alpha, float *t,
                                 const float *T, const float *beta)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= 4 * V) return;
    if (r < 3 * V) {
        const float *row = I + (size_t)r * KA;
        float acc = 0.0f;
        for (int k = 0; k < KA; ++k) acc = fmaf(row[k], alpha[k], acc);
        if (KA) m[r] = m[r] + acc;
    } else {
        const int v = r - 3 * V;
        const float *row = T + (size_t)v * KB;
        float acc = 0.0f;
        for (int k = 0; k < KB; ++k) acc = fmaf(row[k], beta[k], acc);
        if (KB) t[v] = t[v] + acc;
    }
}

}  // namespace tdi
