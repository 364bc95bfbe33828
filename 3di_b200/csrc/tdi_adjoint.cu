// Differentiable render loss and its hand-written adjoint (tdi_batch_loss, tdi_batch_loss_backward).
//
// Loss of a frame: L = -sum_n (gxn_n gxsn_n + gyn_n gysn_n), the negated normalised-gradient
// correlation of 3DI's image term (funcs.cu:842-897, renderer.cu:725-729; the shape fit
// minimises tau_img L plus its barriers), evaluated in FP64 over a frozen set of fragments: the
// visibility (which triangle is sampled at which pixel, and the owner of each pixel) comes from
// the library's raster at the evaluation point; barycentrics, vertex geometry, shading, the
// 15-tap blur and the gradients are recomputed in FP64 from the state. With the visibility held,
// L is a smooth function of (epsilon, tau, u, lambda, L_intensity), and its gradient is exact.
//
// Backward pass (every buffer is recomputed from the state, nothing is kept from the forward):
//   1. per fragment: dL/d(normalised gradients) -> dL/d(gx, gy) through the normalisation ->
//      scattered into dL/d(blurred image) at the four neighbour pixels (FP64 atomics);
//   2. the transposed blur (the taps are symmetric and the border zero, so the transpose is the
//      same separable filter, applied in the opposite order);
//   3. per owner fragment: dL/d(pixel value) through the shading to the light (lambda, L), the
//      translation and rotation (through R^T (lambda - tau)), the object coordinates of its three
//      corners (normal and interpolated point) and the barycentrics, and through those to the
//      projected corners -- scattered to per-vertex accumulators with FP64 atomics, per-frame
//      terms summed per warp first (warp-aggregated atomics);
//   4. per vertex: projected position -> camera coordinates -> rotation, translation and object
//      coordinates; 5. object coordinates -> expression coefficients by the basis-transpose
//      product dL/deps_k = sum_v E[v][:,k] . dL/dP0[v]; 6. dL/dR -> dL/du through dR/du.
// Rotation in FP64: the reference's formula (rotation_header.cu:46-151) evaluated in double.

namespace tdi {

constexpr int AD_THREADS = 256;
constexpr int AD_GLOB = 16;   // per-frame FP64 accumulators: dR[9], dtau[3], dlam[3], dL

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// one atomic per warp for a value every lane contributes to
__device__ __forceinline__ void warp_atomic_add(double *dst, double v)
{
    v = wsum(v);
    if ((threadIdx.x & 31) == 0) atomicAdd(dst, v);
}

__device__ void rotation_d(const float *uf, double *R, double *dR)
{
    const double u[3] = {uf[0], uf[1], uf[2]};
    const double th = sqrt((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
    const double un[3] = {u[0] / th, u[1] / th, u[2] / th};
    auto skew = [](double *S, const double *w) {
        S[0] = 0; S[1] = w[2]; S[2] = -w[1];
        S[3] = -w[2]; S[4] = 0; S[5] = w[0];
        S[6] = w[1]; S[7] = -w[0]; S[8] = 0;
    };
    auto mul = [](const double *A, const double *B, double *C) {
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) C[3 * j + i] = A[i] * B[3 * j] + A[3 + i] * B[3 * j + 1] + A[6 + i] * B[3 * j + 2];
    };
    double Sn[9], Sn2[9], R1[3][9];
    skew(Sn, un);
    mul(Sn, Sn, Sn2);
    const double st = sin(th), cis = 1.0 - cos(th), tinv2 = 1.0 / (th * th);
    for (int i = 0; i < 9; ++i) R[i] = cis * Sn2[i] + ((i % 4 == 0) ? 1.0 : 0.0) + st * Sn[i];
    double IR[9];
    for (int i = 0; i < 9; ++i) IR[i] = ((i % 4 == 0) ? 1.0 : 0.0) - R[i];
    for (int a = 0; a < 3; ++a) {
        skew(R1[a], u);
        for (int i = 0; i < 9; ++i) R1[a][i] *= u[a];
        double R2[9], R3[9];
        const double *c = IR + 3 * a;
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) R2[3 * r + q] = u[r] * c[q];
        for (int i = 0; i < 9; ++i) R1[a][i] += R2[i];
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) R3[3 * r + q] = R1[a][3 * r + q] - R2[3 * q + r];
        mul(R3, R, dR + 9 * a);
        for (int i = 0; i < 9; ++i) dR[9 * a + i] *= tinv2;
    }
}

// Per frame: R, dR/du in FP64 (one thread per frame).
__global__ void k_adj_rot(DModel m, DBatch b, const float *x, int F, double *R64)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    rotation_d(x + (size_t)f * m.KT + m.K + 3, R64 + (size_t)f * 36, R64 + (size_t)f * 36 + 9);
}

// FP64 vertex stage: object coordinates P0 = mean + E eps, camera X = R P0 + tau, projections.
// geo64 [F][V][8]: P0 (3), X (3), xp, yp.
// The same per (frame, vertex), tiled: a block takes AV_V vertices x AV_F frames, stages their
// basis rows and coefficients in shared memory once (instead of every thread reading its
// vertex's rows from L2 for every frame), and each thread forms one vertex of AV_F / 8 frames;
// the fused multiply-add chains over k are the same, in the same order.
constexpr int AV_V = 32, AV_F = 32, AV_FPT = AV_F / 8;

__host__ __device__ __forceinline__ size_t adj_vertex_smem(int KP)
{
    return ((size_t)AV_V * 3 + AV_F) * (size_t)(KP + 1) * sizeof(float);
}

__global__ void __launch_bounds__(256) k_adj_vertex_tiled(DModel m, const float *x, int F, const double *R64,
                                                          const float *cam, double *geo64)
{
    extern __shared__ float avs[];
    const int KP = m.KP, K = m.K, KT = m.KT, W = KP + 1;    // row pitch KP + 1: lanes (vertices) on distinct banks
    float *Es = avs;                                          // [AV_V][3][W]
    float *Xs = Es + (size_t)AV_V * 3 * W;                   // [AV_F][W]
    const int v0 = blockIdx.x * AV_V, f0 = blockIdx.y * AV_F, tid = threadIdx.x;
    for (int i = tid; i < AV_V * 3 * KP; i += 256) {
        const int r = i / KP, k = i - r * KP, v = v0 + r / 3;
        Es[(size_t)r * W + k] = v < m.V ? m.E[(size_t)v0 * 3 * KP + i] : 0.0f;
    }
    for (int i = tid; i < AV_F * KP; i += 256) {
        const int fl = i / KP, k = i - fl * KP, f = f0 + fl;
        Xs[(size_t)fl * W + k] = (f < F && k < K) ? x[(size_t)f * KT + k] : 0.0f;
    }
    __syncthreads();
    const int vl = tid & 31, fg = tid >> 5, v = v0 + vl;
    const float *e0 = Es + (size_t)vl * 3 * W, *e1 = e0 + W, *e2 = e1 + W;
    double acc[AV_FPT][3];
#pragma unroll
    for (int q = 0; q < AV_FPT; ++q) acc[q][0] = acc[q][1] = acc[q][2] = 0.0;
    for (int k = 0; k < K; ++k) {
        const double a0 = e0[k], a1 = e1[k], a2 = e2[k];
#pragma unroll
        for (int q = 0; q < AV_FPT; ++q) {
            const double xv = Xs[(size_t)(fg * AV_FPT + q) * W + k];
            acc[q][0] = fma(a0, xv, acc[q][0]);
            acc[q][1] = fma(a1, xv, acc[q][1]);
            acc[q][2] = fma(a2, xv, acc[q][2]);
        }
    }
    if (v >= m.V) return;
    const double mean[3] = {(double)m.mean[v], (double)m.mean[(size_t)m.V + v], (double)m.mean[2 * (size_t)m.V + v]};
#pragma unroll
    for (int q = 0; q < AV_FPT; ++q) {
        const int f = f0 + fg * AV_FPT + q;
        if (f >= F) break;
        const float *xf = x + (size_t)f * KT;
        double P[3];
        for (int c = 0; c < 3; ++c) P[c] = mean[c] + acc[q][c];
        const double *R = R64 + (size_t)f * 36;
        double X[3];
        for (int i = 0; i < 3; ++i) X[i] = (R[i] * P[0] + R[3 + i] * P[1]) + R[6 + i] * P[2] + (double)xf[K + i];
        const float *cm = cam + (size_t)f * 4;
        double *g = geo64 + ((size_t)f * m.V + v) * 8;
        g[0] = P[0]; g[1] = P[1]; g[2] = P[2];
        g[3] = X[0]; g[4] = X[1]; g[5] = X[2];
        g[6] = (double)cm[0] * X[0] / X[2] + (double)cm[2];
        g[7] = (double)cm[1] * X[1] / X[2] + (double)cm[3];
    }
}

__global__ void k_adj_vertex(DModel m, const float *x, int F, const double *R64, const float *cam, double *geo64)
{
    const int f = blockIdx.y;
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F || v >= m.V) return;
    const float *xf = x + (size_t)f * m.KT;
    double P[3];
    for (int c = 0; c < 3; ++c) {
        const float *e = m.E + ((size_t)v * 3 + c) * m.KP;
        double acc = 0.0;
        for (int k = 0; k < m.K; ++k) acc = fma((double)e[k], (double)xf[k], acc);
        P[c] = (double)m.mean[(size_t)c * m.V + v] + acc;
    }
    const double *R = R64 + (size_t)f * 36;
    double X[3];
    for (int i = 0; i < 3; ++i) X[i] = (R[i] * P[0] + R[3 + i] * P[1]) + R[6 + i] * P[2] + (double)xf[m.K + i];
    const float *cm = cam + (size_t)f * 4;
    double *g = geo64 + ((size_t)f * m.V + v) * 8;
    g[0] = P[0]; g[1] = P[1]; g[2] = P[2];
    g[3] = X[0]; g[4] = X[1]; g[5] = X[2];
    g[6] = (double)cm[0] * X[0] / X[2] + (double)cm[2];
    g[7] = (double)cm[1] * X[1] / X[2] + (double)cm[3];
}

// Barycentrics of sample s in triangle (b, c, a) by Cramer's rule: s - a = alpha (b - a) + beta (c - a)
// (the same values as the reference's dot-product form, funcs.cu:961-977, in exact arithmetic),
// and their derivatives with respect to the three projected corners when d != nullptr:
// d[0..5] = dalpha/d(b, c, a) (x, y each), d[6..11] = dbeta/d(b, c, a).
__device__ __forceinline__ void bary_d(const double *pb, const double *pc, const double *pa, double sx, double sy,
                                       double &al, double &be, double *d)
{
    const double v0x = pb[0] - pa[0], v0y = pb[1] - pa[1], v1x = pc[0] - pa[0], v1y = pc[1] - pa[1];
    const double v2x = sx - pa[0], v2y = sy - pa[1];
    const double D = v0x * v1y - v0y * v1x;
    al = (v2x * v1y - v2y * v1x) / D;
    be = (v0x * v2y - v0y * v2x) / D;
    if (!d) return;
    // dD/dv0 = (v1y, -v1x), dD/dv1 = (-v0y, v0x)
    const double a0x = -al * v1y / D, a0y = al * v1x / D;                            // dalpha/dv0
    const double a1x = (-v2y + al * v0y) / D, a1y = (v2x - al * v0x) / D;            // dalpha/dv1
    const double a2x = v1y / D, a2y = -v1x / D;                                       // dalpha/dv2
    const double b0x = (v2y - be * v1y) / D, b0y = (-v2x + be * v1x) / D;            // dbeta/dv0
    const double b1x = be * v0y / D, b1y = -be * v0x / D;                             // dbeta/dv1
    const double b2x = -v0y / D, b2y = v0x / D;                                       // dbeta/dv2
    d[0] = a0x; d[1] = a0y; d[2] = a1x; d[3] = a1y; d[4] = -(a0x + a1x + a2x); d[5] = -(a0y + a1y + a2y);
    d[6] = b0x; d[7] = b0y; d[8] = b1x; d[9] = b1y; d[10] = -(b0x + b1x + b2x); d[11] = -(b0y + b1y + b2y);
}

struct AdjFrame {                 // a frame's inputs to the FP64 render
    const double *geo, *R;        // [V][8], [9]
    const float *x, *lam;         // state [KT], light [3]
    float L;
    int x0, y0, N;
    const Fragment *fr;
};

__device__ __forceinline__ AdjFrame adj_frame(const DModel &m, const DBatch &b, const float *x, const float *lam,
                                              const float *Lint, const double *geo64, const double *R64, int f)
{
    AdjFrame a;
    a.geo = geo64 + (size_t)f * m.V * 8;
    a.R = R64 + (size_t)f * 36;
    a.x = x + (size_t)f * m.KT;
    a.lam = lam + (size_t)f * 3;
    a.L = Lint[f];
    a.x0 = b.x0y0[2 * f];
    a.y0 = b.x0y0[2 * f + 1];
    a.N = b.ctl[f].N;
    a.fr = b.frag + (size_t)f * NMAX;
    return a;
}

// FP64 shading of the owner fragments painted into a zero image (fill_diffuse_component...,
// newfuncs.cu:18-167, and fill_tex_im1, funcs.cu:800-817).
__global__ void k_adj_shade(DModel m, DBatch b, const float *x, const float *lam, const float *Lint, int F,
                            const double *geo64, const double *R64, double *img)
{
    const int f = blockIdx.y;
    if (f >= F) return;
    const AdjFrame a = adj_frame(m, b, x, lam, Lint, geo64, R64, f);
    double *im = img + (size_t)f * NPIX;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.N; n += gridDim.x * blockDim.x) {
        const Fragment fr = a.fr[n];
        if (!(fr.pix_owner >> 31)) continue;
        const int pix = fr.pix_owner & 0xFFFF, tri = fr.tri;
        const int ib = m.tl[tri], ic = m.tl[m.T + tri], ia = m.tl[2 * m.T + tri];
        const double *gb = a.geo + (size_t)ib * 8, *gc = a.geo + (size_t)ic * 8, *ga = a.geo + (size_t)ia * 8;
        double al, be;
        bary_d(gb + 6, gc + 6, ga + 6, (double)(a.x0 + (pix >> 8)), (double)(a.y0 + (pix & 255)), al, be, nullptr);
        const double gm = 1.0 - al - be;
        double v[3], w[3], nr[3];
        for (int c = 0; c < 3; ++c) { v[c] = gb[c] - ga[c]; w[c] = gc[c] - ga[c]; }
        nr[0] = v[1] * w[2] - v[2] * w[1]; nr[1] = v[2] * w[0] - v[0] * w[2]; nr[2] = v[0] * w[1] - v[1] * w[0];
        const double nn = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
        double Id = 0.0;
        for (int k = 0; k < 3; ++k) {
            double q = 0.0;
            for (int j = 0; j < 3; ++j) q += a.R[3 * k + j] * ((double)a.lam[j] - (double)a.x[m.K + j]);
            const double p = gb[k] * al + gc[k] * be + ga[k] * gm;
            Id += nr[k] / nn * (q - p);
        }
        const double t = (double)m.tex[ib] * al + (double)m.tex[ic] * be + (double)m.tex[ia] * gm;
        im[pix] = t + (double)a.L * t * Id;
    }
}

// FP64 separable blur pass (the 15 taps of the fit, zero border): along y (dir 0) or x (dir 1).
__global__ void k_adj_blur(const double *src, double *dst, Cfg c, int F, int dir)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)F * NPIX) return;
    const size_t f = i / NPIX;
    const int p = (int)(i - f * NPIX), xx = p >> 8, yy = p & 255;
    const double *s = src + f * NPIX;
    double acc = 0.0;
    for (int j = -KRAD; j <= KRAD; ++j) {
        const int u = (dir == 0 ? yy : xx) + j;
        if (u < 0 || u >= DIM) continue;
        acc += (double)c.taps[KRAD - j] * s[dir == 0 ? xx * DIM + u : u * DIM + yy];
    }
    dst[i] = acc;
}

// FP32 crops to FP64 (the target before its blur).
__global__ void k_adj_widen(const float *src, double *dst, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (double)src[i];
}

// Normalised central-difference gradients at every fragment (fill_grads, funcs.cu:842-897) of
// the blurred render B and target T; loss sums into loss[f]; with adjB, the adjoint of the
// gradients scattered into dL/dB (gloss[f] scales the frame's loss gradient).
__global__ void k_adj_grad(DBatch b, int F, const double *B, const double *T, double *loss, const double *gloss,
                           double *adjB)
{
    const int f = blockIdx.y;
    if (f >= F) return;
    const int N = b.ctl[f].N;
    const Fragment *frs = b.frag + (size_t)f * NMAX;
    const double *Bf = B + (size_t)f * NPIX, *Tf = T + (size_t)f * NPIX;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        const int p = frs[n].pix_owner & 0xFFFF, x = p >> 8, y = p & 255;
        const int kr = x < DIM - 1 ? p + DIM : 0, kl = x > 0 ? p - DIM : 0;
        const int kb = y < DIM - 1 ? p + 1 : 0, ka = y > 0 ? p - 1 : 0;
        const double gx = 0.5 * (Bf[kr] - Bf[kl]), gy = 0.5 * (Bf[kb] - Bf[ka]);
        const double r = sqrt(4.0 * gx * gx + 4.0 * gy * gy), h = 1e-16 + r;
        const double sx = 0.5 * (Tf[kr] - Tf[kl]), sy = 0.5 * (Tf[kb] - Tf[ka]);
        const double hs = 1e-16 + sqrt(4.0 * sx * sx + 4.0 * sy * sy);
        const double sxn = 2.0 * sx / hs, syn = 2.0 * sy / hs;
        part += -((2.0 * gx / h) * sxn + (2.0 * gy / h) * syn);
        if (adjB) {
            const double gl = gloss[f];
            const double dgxn = -gl * sxn, dgyn = -gl * syn;         // dL/d(2 gx / h), dL/d(2 gy / h)
            const double dh = r > 0.0 ? 1.0 / r : 0.0;
            const double hx = 4.0 * gx * dh, hy = 4.0 * gy * dh;     // dh/dgx, dh/dgy
            const double dgx = dgxn * (2.0 / h - 2.0 * gx * hx / (h * h)) + dgyn * (-2.0 * gy * hx / (h * h));
            const double dgy = dgxn * (-2.0 * gx * hy / (h * h)) + dgyn * (2.0 / h - 2.0 * gy * hy / (h * h));
            double *A = adjB + (size_t)f * NPIX;
            atomicAdd(A + kr, 0.5 * dgx);
            atomicAdd(A + kl, -0.5 * dgx);
            atomicAdd(A + kb, 0.5 * dgy);
            atomicAdd(A + ka, -0.5 * dgy);
        }
    }
    warp_atomic_add(loss + f, part);
}

// Adjoint of the shading of the owner fragments: dL/dpixel -> light, pose (through R^T (lam - tau)),
// object coordinates of the corners (normal, interpolated point) and projected corners
// (barycentrics). Per-vertex terms by FP64 atomics, per-frame terms summed per warp.
__global__ void k_adj_frag_back(DModel m, DBatch b, const float *x, const float *lam, const float *Lint, int F,
                                const double *geo64, const double *R64, const double *adjI, double *dP0, double *dpos,
                                double *glob)
{
    const int f = blockIdx.y;
    if (f >= F) return;
    const AdjFrame a = adj_frame(m, b, x, lam, Lint, geo64, R64, f);
    const double *AI = adjI + (size_t)f * NPIX;
    double acc[AD_GLOB];
#pragma unroll
    for (int i = 0; i < AD_GLOB; ++i) acc[i] = 0.0;
    double dl[3];
    for (int j = 0; j < 3; ++j) dl[j] = (double)a.lam[j] - (double)a.x[m.K + j];
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.N; n += gridDim.x * blockDim.x) {
        const Fragment fr = a.fr[n];
        if (!(fr.pix_owner >> 31)) continue;
        const int pix = fr.pix_owner & 0xFFFF, tri = fr.tri;
        const double dI = AI[pix];
        if (dI == 0.0) continue;
        const int iv[3] = {m.tl[tri], m.tl[m.T + tri], m.tl[2 * m.T + tri]};        // b, c, a
        const double *gb = a.geo + (size_t)iv[0] * 8, *gc = a.geo + (size_t)iv[1] * 8, *ga = a.geo + (size_t)iv[2] * 8;
        double al, be, db[12];
        bary_d(gb + 6, gc + 6, ga + 6, (double)(a.x0 + (pix >> 8)), (double)(a.y0 + (pix & 255)), al, be, db);
        const double gm = 1.0 - al - be;
        double v[3], w[3], nr[3], nh[3], q[3], p[3];
        for (int c = 0; c < 3; ++c) { v[c] = gb[c] - ga[c]; w[c] = gc[c] - ga[c]; }
        nr[0] = v[1] * w[2] - v[2] * w[1]; nr[1] = v[2] * w[0] - v[0] * w[2]; nr[2] = v[0] * w[1] - v[1] * w[0];
        const double nn = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
        double Id = 0.0;
        for (int k = 0; k < 3; ++k) {
            nh[k] = nr[k] / nn;
            q[k] = 0.0;
            for (int j = 0; j < 3; ++j) q[k] += a.R[3 * k + j] * dl[j];
            p[k] = gb[k] * al + gc[k] * be + ga[k] * gm;
            Id += nh[k] * (q[k] - p[k]);
        }
        const double tb = m.tex[iv[0]], tc = m.tex[iv[1]], ta = m.tex[iv[2]];
        const double t = tb * al + tc * be + ta * gm, L = a.L;
        const double dt = dI * (1.0 + L * Id), dId = dI * L * t;
        acc[15] += dI * t * Id;                                          // dL/dL_intensity
        double dal = dt * (tb - ta), dbe = dt * (tc - ta);
        double dn[3], dP[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int k = 0; k < 3; ++k) {
            dn[k] = dId * (q[k] - p[k]);
            const double dq = dId * nh[k], dp = -dId * nh[k];
            for (int j = 0; j < 3; ++j) {
                acc[3 * k + j] += dq * dl[j];                            // dR[3k + j]
                const double dd = dq * a.R[3 * k + j];
                acc[12 + j] += dd;                                       // dlambda_j
                acc[9 + j] -= dd;                                        // dtau_j
            }
            dal += dp * (gb[k] - ga[k]);
            dbe += dp * (gc[k] - ga[k]);
            dP[0][k] += al * dp; dP[1][k] += be * dp; dP[2][k] += gm * dp;
        }
        const double nd = nh[0] * dn[0] + nh[1] * dn[1] + nh[2] * dn[2];
        double dnr[3];
        for (int k = 0; k < 3; ++k) dnr[k] = (dn[k] - nh[k] * nd) / nn;
        // nr = v x w: dL/dv = w x dnr, dL/dw = dnr x v
        const double dv[3] = {w[1] * dnr[2] - w[2] * dnr[1], w[2] * dnr[0] - w[0] * dnr[2], w[0] * dnr[1] - w[1] * dnr[0]};
        const double dw[3] = {dnr[1] * v[2] - dnr[2] * v[1], dnr[2] * v[0] - dnr[0] * v[2], dnr[0] * v[1] - dnr[1] * v[0]};
        for (int k = 0; k < 3; ++k) {
            dP[0][k] += dv[k];
            dP[1][k] += dw[k];
            dP[2][k] -= dv[k] + dw[k];
        }
        double *P0f = dP0 + (size_t)f * m.V * 3, *pf = dpos + (size_t)f * m.V * 2;
        for (int c = 0; c < 3; ++c) {
            for (int k = 0; k < 3; ++k) atomicAdd(P0f + (size_t)iv[c] * 3 + k, dP[c][k]);
            atomicAdd(pf + (size_t)iv[c] * 2 + 0, dal * db[2 * c] + dbe * db[6 + 2 * c]);
            atomicAdd(pf + (size_t)iv[c] * 2 + 1, dal * db[2 * c + 1] + dbe * db[6 + 2 * c + 1]);
        }
    }
#pragma unroll
    for (int i = 0; i < AD_GLOB; ++i) warp_atomic_add(glob + (size_t)f * AD_GLOB + i, acc[i]);
}

// Per vertex: dL/d(xp, yp) -> camera coordinates -> translation, rotation and object coordinates
// (added to dP0 in place).
__global__ void k_adj_vertex_back(DModel m, int F, const double *geo64, const double *R64, const float *cam,
                                  const double *dpos, double *dP0, double *glob)
{
    const int f = blockIdx.y;
    if (f >= F) return;
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) acc[i] = 0.0;
    if (v < m.V) {
        const double *g = geo64 + ((size_t)f * m.V + v) * 8, *R = R64 + (size_t)f * 36;
        const float *cm = cam + (size_t)f * 4;
        const double gx = dpos[((size_t)f * m.V + v) * 2], gy = dpos[((size_t)f * m.V + v) * 2 + 1];
        const double X = g[3], Y = g[4], Z = g[5];
        const double gc[3] = {gx * cm[0] / Z, gy * cm[1] / Z, -(gx * cm[0] * X + gy * cm[1] * Y) / (Z * Z)};
        double *P = dP0 + ((size_t)f * m.V + v) * 3;
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int i = 0; i < 3; ++i) {
                acc[i + 3 * j] += gc[i] * g[j];                          // dR[i + 3j] (X = R P0 + tau)
                s += gc[i] * R[i + 3 * j];
            }
            P[j] += s;
            acc[9 + j] += gc[j];                                         // dtau_j
        }
    }
    // the per-fragment rotation terms are indexed by q_k = sum_j R[3k + j] (lam - tau)_j: both
    // index the same storage, so they add up entry by entry; summed per warp, then per block,
    // one atomic per block and entry
    __shared__ double s_acc[8][12];
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const double w = wsum(acc[i]);
        if ((threadIdx.x & 31) == 0) s_acc[threadIdx.x >> 5][i] = w;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_acc[w][threadIdx.x];
        atomicAdd(glob + (size_t)f * AD_GLOB + threadIdx.x, t);
    }
}

// Basis-transpose product dL/deps_k = sum_v sum_c E[v][c][k] dL/dP0[v][c] over a tile of vertices.
constexpr int AD_VT = 256;
// A block takes AD_VT vertices x AE_F frames (threads = expression columns), so that each
// basis row is read once per AE_F frames; per frame and column the vertex terms are summed in
// vertex order, the block's partial added with one atomic.
constexpr int AE_F = 16;

__global__ void k_adj_eps(DModel m, int F, const double *dP0, double *geps)
{
    const int k = threadIdx.x, f0 = blockIdx.y * AE_F;
    const int v0 = blockIdx.x * AD_VT, v1 = min(m.V, v0 + AD_VT);
    const bool live = k < m.K;
    double acc[AE_F];
#pragma unroll
    for (int q = 0; q < AE_F; ++q) acc[q] = 0.0;
    for (int v = v0; v < v1; ++v) {
        const float *e = m.E + (size_t)v * 3 * m.KP + (live ? k : 0);
        const double e0 = e[0], e1 = e[m.KP], e2 = e[2 * m.KP];
#pragma unroll
        for (int q = 0; q < AE_F; ++q) {
            const int f = f0 + q;
            if (f >= F) break;
            const double *P = dP0 + ((size_t)f * m.V + v) * 3;
            acc[q] += e0 * P[0] + e1 * P[1] + e2 * P[2];
        }
    }
    if (!live) return;
#pragma unroll
    for (int q = 0; q < AE_F; ++q) {
        const int f = f0 + q;
        if (f >= F) break;
        atomicAdd(geps + (size_t)f * m.K + k, acc[q]);
    }
}

// Gradients out: x [F][K+6] (epsilon, tau, u through dR/du), lambda [F][3], L [F].
__global__ void k_adj_final(DModel m, int F, const double *R64, const double *glob, const double *geps, double *gx,
                            double *glam, double *gL)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const double *G = glob + (size_t)f * AD_GLOB, *dR = R64 + (size_t)f * 36 + 9;
    double *o = gx + (size_t)f * m.KT;
    for (int k = 0; k < m.K; ++k) o[k] = geps[(size_t)f * m.K + k];
    for (int j = 0; j < 3; ++j) o[m.K + j] = G[9 + j];
    for (int a = 0; a < 3; ++a) {
        double s = 0.0;
        for (int i = 0; i < 9; ++i) s += G[i] * dR[9 * a + i];
        o[m.K + 3 + a] = s;
    }
    if (glam)
        for (int j = 0; j < 3; ++j) glam[(size_t)f * 3 + j] = G[12 + j];
    if (gL) gL[f] = G[15];
}

// The caller's states [F][K+6] into the batch's evaluation states (pitch KTP).
__global__ void k_adj_set_x(DModel m, DBatch b, const float *x, int F)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F * m.KT) return;
    const int f = i / m.KT, a = i - f * m.KT;
    b.x[(size_t)f * m.KTP + a] = x[i];
    b.x_ls[(size_t)f * m.KTP + a] = x[i];
}

}  // namespace tdi
