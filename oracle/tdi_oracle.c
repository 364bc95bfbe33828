/*
 * CPU oracle for the 3DI per-frame fitting path -- TEST INFRASTRUCTURE ONLY (see
 * tdi_oracle.h). Restates, operation by operation, the reference CUDA sources of
 * Computational-Psychiatry/3DI; each function names the file:line it follows.
 * Parity is pinned to the reference's own kernels, built from its sources by ref.mk into
 * _ref/ and compared stage by stage in tests/test_ref_pinning.py.
 *
 * Arithmetic definitions (identical in the product's CUDA kernels):
 *  - elementwise formulas: IEEE arithmetic in REAL, no FMA contraction, the operand order
 *    of the reference source (gcc -ffp-contract=off here, nvcc -fmad=false there);
 *  - where the reference calls cuBLAS (SGEMV for basis x coefficients, SGEMM/SDOT for
 *    sums over fragments or landmarks) the order is unspecified; this file defines
 *    SGEMV as a sequential fused multiply-add over k starting from 0, then added to the
 *    mean, and accumulates all other sums in double;
 *  - sin, cos and log are evaluated in double and rounded to REAL;
 *  - the Cholesky factor/solve is FP64 as in the reference (solver.h:70-105).
 */
#include "tdi_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef TDI_REAL_DOUBLE
typedef double real;
#define RSQRT(x) sqrt(x)
#define RFMA(a, b, c) fma((a), (b), (c))
#define RFABS(x) fabs(x)
#else
typedef float real;
#define RSQRT(x) sqrtf(x)
#define RFMA(a, b, c) fmaf((a), (b), (c))
#define RFABS(x) fabsf(x)
#endif
#define RSIN(x) ((real)sin((double)(x)))
#define RCOS(x) ((real)cos((double)(x)))
#define RLOG(x) ((real)log((double)(x)))

#define NL O_NL
#define DIM O_DIM
#define NPIX O_NPIX
#define NTMP O_NTMP
#define KRAD 7

/* ------------------------------------------------------------------------------------ */
/* Rotation R(u) and dR/du_i: rotation_header.cu:46-151 (fill_theta_etc), helpers :22-200 */

static void mul33(const real *A, const real *B, real *C)   /* multiplyAB_3x3, :24-37 */
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

static void skew(real *S, const real *u)                   /* fill_skew_matrix_dev */
{
    S[0] = 0; S[1] = u[2]; S[2] = -u[1];
    S[3] = -u[2]; S[4] = 0; S[5] = u[0];
    S[6] = u[1]; S[7] = -u[0]; S[8] = 0;
}

void o_rotation(const real *u, real *R, real *dR /* [3][9] or NULL */)
{
    real theta = RSQRT((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
    real un[3] = {u[0] / theta, u[1] / theta, u[2] / theta};
    real R1[3][9], Sn[9], Sn2[9];
    skew(R1[0], u); skew(R1[1], u); skew(R1[2], u);
    skew(Sn, un);
    real st = RSIN(theta);
    real cis = (real)1 - RCOS(theta);
    real tinv2 = (real)1 / (theta * theta);
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i < 9; ++i) R1[a][i] *= u[a];
    mul33(Sn, Sn, Sn2);
    for (int i = 0; i < 9; ++i) {
        if (i == 0 || i == 4 || i == 8)
            R[i] = (cis * Sn2[i] + (real)1) + st * Sn[i];
        else
            R[i] = cis * Sn2[i] + st * Sn[i];
    }
    if (!dR) return;
    real IR[9];
    for (int i = 0; i < 9; ++i) IR[i] = R[i] * (real)-1;
    IR[0] += 1; IR[4] += 1; IR[8] += 1;
    for (int a = 0; a < 3; ++a) {
        real R2[9], R3[9];
        const real *c = IR + 3 * a;        /* column a of I - R */
        R2[0] = u[0] * c[0]; R2[1] = u[0] * c[1]; R2[2] = u[0] * c[2];
        R2[3] = u[1] * c[0]; R2[4] = u[1] * c[1]; R2[5] = u[1] * c[2];
        R2[6] = u[2] * c[0]; R2[7] = u[2] * c[1]; R2[8] = u[2] * c[2];
        for (int i = 0; i < 9; ++i) R1[a][i] += R2[i];     /* sum_AB_3x3_inplace */
        R3[0] = R1[a][0] - R2[0]; R3[1] = R1[a][1] - R2[3]; R3[2] = R1[a][2] - R2[6];
        R3[3] = R1[a][3] - R2[1]; R3[4] = R1[a][4] - R2[4]; R3[5] = R1[a][5] - R2[7];
        R3[6] = R1[a][6] - R2[2]; R3[7] = R1[a][7] - R2[5]; R3[8] = R1[a][8] - R2[8];
        mul33(R3, R, dR + 9 * a);
        for (int i = 0; i < 9; ++i) dR[9 * a + i] *= tinv2;
    }
}

/* ------------------------------------------------------------------------------------ */
/* Vertex stage: Renderer::compute_nonrigid_shape2 (renderer.cu:806-861) with
 * view_transform_3d_pts_and_render_2d (funcs.cu:395-453). geo = [8][V]:
 * X0, Y0, Z0 (object), X, Y, Z (camera), xp, yp. Returns the face-size check result. */

int o_vertex_stage(const o_model *m, const real *eps, const real *R, const real *tau,
                   const float *cam, float ref_face_size, real *geo)
{
    const int V = m->V, K = m->K;
    real *X0 = geo, *Y0 = geo + V, *Z0 = geo + 2 * V;
    real *X = geo + 3 * V, *Y = geo + 4 * V, *Z = geo + 5 * V, *xp = geo + 6 * V, *yp = geo + 7 * V;
    const real phix = cam[0], phiy = cam[1], cx = cam[2], cy = cam[3];
    for (int v = 0; v < V; ++v) {
        real P[3];
        for (int c = 0; c < 3; ++c) {
            const float *e = m->E + ((size_t)v * 3 + c) * K;
            real acc = 0;
            for (int k = 0; k < K; ++k) acc = RFMA((real)e[k], eps[k], acc);
            P[c] = (real)m->mean[c * V + v] + acc;
        }
        X0[v] = P[0]; Y0[v] = P[1]; Z0[v] = P[2];
        real X3 = ((R[0] * P[0] + R[3] * P[1]) + R[6] * P[2]) + tau[0];
        real Y3 = ((R[1] * P[0] + R[4] * P[1]) + R[7] * P[2]) + tau[1];
        real Z3 = ((R[2] * P[0] + R[5] * P[1]) + R[8] * P[2]) + tau[2];
        X[v] = X3; Y[v] = Y3; Z[v] = Z3;
        xp[v] = (phix * X3) / Z3 + cx;
        yp[v] = (phiy * Y3) / Z3 + cy;
    }
    /* renderer.cu:838-857: inter-ocular and eye-mouth distances vs 2*REF_FACE_SIZE */
    const int *L = m->lis;
    real d_iod = RFABS(xp[L[9]] - xp[L[0]]);
    real d_lem = RFABS(yp[L[0]] - yp[L[40]]);
    real d_rem = RFABS(yp[L[9]] - yp[L[40]]);
    double lim = (double)ref_face_size * 2;
    return !((double)d_iod > lim || (double)d_lem > lim || (double)d_rem > lim);
}

/* ------------------------------------------------------------------------------------ */
/* Visibility: get_pixels_to_render + atomicMinFloat (funcs.cu:900-1010), keep_only_minZ
 * (:1016-1029) and thrust::remove_if(is_zero) (renderer.cu:650-680).
 * Fragments of a triangle occupy slots r*T + tri (r < NTMP) in bounding-box order (x
 * outer, y inner); a fragment survives iff its depth (camera Z of the triangle's first
 * vertex) equals the per-pixel minimum; survivors keep slot order; slot 0 is always
 * dropped. The pixel owner among depth ties is the smallest triangle id (the packed
 * (depth bits, triangle id) minimum); it paints the image only if it survived. */

typedef struct {
    int32_t n;
    int32_t *slot;
    int32_t *tri;
    uint16_t *pix;
    float *al, *be, *ga;
    uint8_t *owner;
} o_frags;

static inline uint16_t to_u16_floor(float v, uint32_t *flags)
{
    float f = floorf(v);
    if (!(f >= 0.0f) || f > 65535.0f) { *flags |= O_FLAG_OUT_OF_DOMAIN; return f > 0 ? 65535 : 0; }
    return (uint16_t)f;
}

static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

int o_raster(const o_model *m, const float *xp, const float *yp, const float *Zc,
             int x0, int y0, o_frags *out, uint32_t *flags)
{
    const int T = m->T;
    const int32_t *tl = m->tl;
    uint16_t *fpix = (uint16_t *)malloc(sizeof(uint16_t) * 4 * (size_t)T);
    float *fal = (float *)malloc(sizeof(float) * 4 * (size_t)T);
    float *fbe = (float *)malloc(sizeof(float) * 4 * (size_t)T);
    uint8_t *cnt = (uint8_t *)calloc((size_t)T, 1);
    float *zmin = (float *)malloc(sizeof(float) * NPIX);
    uint64_t *kmin = (uint64_t *)malloc(sizeof(uint64_t) * NPIX);
    for (int p = 0; p < NPIX; ++p) { zmin[p] = 3.40282347e38f; kmin[p] = ~0ull; }

    for (int idx = 0; idx < T; ++idx) {
        const int ib = tl[idx], ic = tl[T + idx], ia = tl[2 * T + idx];
        const float bx = xp[ib], cx = xp[ic], ax = xp[ia];
        const float by = yp[ib], cy = yp[ic], ay = yp[ia];
        const float Z = Zc[ib];
        const float xhi = ceilf(fmaxf(fmaxf(bx, cx), ax));
        const float yhi = ceilf(fmaxf(fmaxf(by, cy), ay));
        const uint16_t xlo = to_u16_floor(fminf(fminf(bx, cx), ax), flags);
        const uint16_t ylo = to_u16_floor(fminf(fminf(by, cy), ay), flags);
        if (!(xhi <= 65535.0f && yhi <= 65535.0f)) { *flags |= O_FLAG_OUT_OF_DOMAIN; cnt[idx] = 0; continue; }
        /* a box larger than the crop only comes from a vertex near the camera plane; the
           reference would walk all of it -- skipped and flagged */
        if ((xhi - (float)xlo) * (yhi - (float)ylo) > 65536.0f) { *flags |= O_FLAG_OUT_OF_DOMAIN; cnt[idx] = 0; continue; }
        int ridx = 0;
        for (uint16_t x = xlo; (float)x < xhi && ridx < NTMP; ++x) {
            for (uint16_t y = ylo; (float)y < yhi && ridx < NTMP; ++y) {
                float v0x = bx - ax, v1x = cx - ax, v2x = (float)x - ax;
                float v0y = by - ay, v1y = cy - ay, v2y = (float)y - ay;
                float d00 = v0x * v0x + v0y * v0y;
                float d01 = v0x * v1x + v0y * v1y;
                float d11 = v1x * v1x + v1y * v1y;
                float d20 = v0x * v2x + v0y * v2y;
                float d21 = v1x * v2x + v1y * v2y;
                float denom = d00 * d11 - d01 * d01;
                float alpha = (d11 * d20 - d01 * d21) / denom;
                float beta = (d00 * d21 - d01 * d20) / denom;
                if (alpha > 0 && beta > 0 && (alpha + beta <= 1)) {
                    size_t s = (size_t)ridx * T + idx;
                    int px = ((int)y - y0) + ((int)x - x0) * DIM;
                    if (px < 0 || px >= NPIX) *flags |= O_FLAG_OUT_OF_DOMAIN;
                    uint16_t pix = (uint16_t)px;
                    fpix[s] = pix; fal[s] = alpha; fbe[s] = beta;
                    if (Z < zmin[pix]) zmin[pix] = Z;
                    uint64_t key = ((uint64_t)fbits(Z) << 32) | (uint32_t)idx;
                    if (key < kmin[pix]) kmin[pix] = key;
                    ridx++;
                }
            }
        }
        cnt[idx] = (uint8_t)ridx;
        if (ridx && !(Z > 0.0f)) *flags |= O_FLAG_OUT_OF_DOMAIN;
    }
    int n = 0;
    int bx0 = 1 << 30, bx1 = -1, by0 = 1 << 30, by1 = -1;
    for (int r = 0; r < NTMP; ++r) {
        for (int idx = 0; idx < T; ++idx) {
            if (cnt[idx] <= r) continue;
            size_t s = (size_t)r * T + idx;
            if (s == 0) continue;                                   /* remove_if drops slot 0 */
            const uint16_t pix = fpix[s];
            if (Zc[tl[idx]] != zmin[pix]) continue;
            if (out) {
                out->slot[n] = (int32_t)s;
                out->tri[n] = idx;
                out->pix[n] = pix;
                out->al[n] = fal[s];
                out->be[n] = fbe[s];
                out->ga[n] = (1 - fal[s]) - fbe[s];
                uint64_t key = ((uint64_t)fbits(Zc[tl[idx]]) << 32) | (uint32_t)idx;
                out->owner[n] = (key == kmin[pix]);
            }
            {
                const int px = pix >> 8, py = pix & 255;
                if (px < bx0) bx0 = px;
                if (px > bx1) bx1 = px;
                if (py < by0) by0 = py;
                if (py > by1) by1 = py;
            }
            n++;
        }
    }
    if (out) out->n = n;
    free(fpix); free(fal); free(fbe); free(cnt); free(zmin); free(kmin);
    if (n < 1000 || n > 52000) *flags |= O_FLAG_RENDER_SKIPPED;
    if (n > 25600) *flags |= O_FLAG_OUT_OF_DOMAIN;
    if (bx1 >= 0 && (bx0 < 1 || bx1 > DIM - 2 || by0 < 1 || by1 > DIM - 2)) *flags |= O_FLAG_OUT_OF_DOMAIN;
    return n;
}

/* ------------------------------------------------------------------------------------ */
/* Shading of each fragment: fill_diffuse_component_and_populate_texture_and_shape
 * (newfuncs.cu:18-167). sh = [14][N]: shaded, Id, dIdL, dIdlam_raw[3], p[3], v[3],
 * inv_vz, inv_vz2. */

enum { SH_TEX = 0, SH_ID, SH_DIDL, SH_DLAM, SH_P = SH_DLAM + 3, SH_V = SH_P + 3,
       SH_IVZ = SH_V + 3, SH_IVZ2, SH_N };

static void shade(const o_model *m, const real *geo, const o_frags *fr, const real *R,
                  const real *tau, const real *lam, real Lint, real *sh, int N)
{
    const int V = m->V, T = m->T;
    const real *X0 = geo, *Y0 = geo + V, *Z0 = geo + 2 * V;
    const real *X = geo + 3 * V, *Y = geo + 4 * V, *Z = geo + 5 * V;
    for (int n = 0; n < fr->n; ++n) {
        const int tri = fr->tri[n];
        const int ib = m->tl[tri], ic = m->tl[T + tri], ia = m->tl[2 * T + tri];
        const real al = fr->al[n], be = fr->be[n], ga = fr->ga[n];
        real b0x = X0[ib], b0y = Y0[ib], b0z = Z0[ib];
        real c0x = X0[ic], c0y = Y0[ic], c0z = Z0[ic];
        real a0x = X0[ia], a0y = Y0[ia], a0z = Z0[ia];
        real n_vx = b0x - a0x, n_vy = b0y - a0y, n_vz = b0z - a0z;
        real n_wx = c0x - a0x, n_wy = c0y - a0y, n_wz = c0z - a0z;
        real nrx = n_vy * n_wz - n_vz * n_wy;
        real nry = n_vz * n_wx - n_vx * n_wz;
        real nrz = n_vx * n_wy - n_vy * n_wx;
        real normn = RSQRT((nrx * nrx + nry * nry) + nrz * nrz);
        real nn0 = nrx / normn, nn1 = nry / normn, nn2 = nrz / normn;
        real s0 = (b0x * al + c0x * be) + a0x * ga;
        real s1 = (b0y * al + c0y * be) + a0y * ga;
        real s2 = (b0z * al + c0z * be) + a0z * ga;
        real d0 = lam[0] - tau[0], d1 = lam[1] - tau[1], d2 = lam[2] - tau[2];
        real Id = (nn0 * ((R[0] * d0 + R[1] * d1) + R[2] * d2)
                   + nn1 * ((R[3] * d0 + R[4] * d1) + R[5] * d2))
                  + nn2 * ((R[6] * d0 + R[7] * d1) + R[8] * d2);
        Id = Id - ((nn0 * s0 + nn1 * s1) + nn2 * s2);
        real t = ((real)m->tex[ib] * al + (real)m->tex[ic] * be) + (real)m->tex[ia] * ga;
        real Lt = Lint * t;
        sh[SH_TEX * N + n] = t + Lt * Id;
        sh[SH_ID * N + n] = Id;
        sh[SH_DIDL * N + n] = t * Id;
        sh[(SH_DLAM + 0) * N + n] = Lt * nn0;
        sh[(SH_DLAM + 1) * N + n] = Lt * nn1;
        sh[(SH_DLAM + 2) * N + n] = Lt * nn2;
        sh[(SH_P + 0) * N + n] = s0;
        sh[(SH_P + 1) * N + n] = s1;
        sh[(SH_P + 2) * N + n] = s2;
        real vx = (X[ib] * al + X[ic] * be) + X[ia] * ga;
        real vy = (Y[ib] * al + Y[ic] * be) + Y[ia] * ga;
        real vz = (Z[ib] * al + Z[ic] * be) + Z[ia] * ga;
        sh[(SH_V + 0) * N + n] = vx;
        sh[(SH_V + 1) * N + n] = vy;
        sh[(SH_V + 2) * N + n] = vz;
        real ivz = (real)1 / vz;
        sh[SH_IVZ * N + n] = ivz;
        sh[SH_IVZ2 * N + n] = ivz * ivz;
    }
}

/* 15-tap separable Gaussian, zero padding: convolutionRowsKernel (newfuncs.cu:539-595) along
 * the contiguous index, then convolutionColumnsKernel (:634-690) along the strided one. */
static void blur(const float *taps, const real *src, real *tmp, real *dst)
{
    for (int x = 0; x < DIM; ++x)
        for (int y = 0; y < DIM; ++y) {
            real s = 0;
            for (int j = -KRAD; j <= KRAD; ++j) {
                int yy = y + j;
                real v = (yy >= 0 && yy < DIM) ? src[x * DIM + yy] : (real)0;
                s = s + (real)taps[KRAD - j] * v;
            }
            tmp[x * DIM + y] = s;
        }
    for (int x = 0; x < DIM; ++x)
        for (int y = 0; y < DIM; ++y) {
            real s = 0;
            for (int j = -KRAD; j <= KRAD; ++j) {
                int xx = x + j;
                real v = (xx >= 0 && xx < DIM) ? tmp[xx * DIM + y] : (real)0;
                s = s + (real)taps[KRAD - j] * v;
            }
            dst[x * DIM + y] = s;
        }
}

/* fill_grads (funcs.cu:842-897) for one image at one pixel. */
static inline void pixel_grad(const real *im, uint16_t ks, real *gx, real *gy, real *gxn, real *gyn, real *h)
{
    uint16_t y = ks % DIM, x = ks / DIM;
    uint16_t kr = (x < DIM - 1) ? (uint16_t)((x + 1) * DIM + y) : 0;
    uint16_t kl = (x > 0) ? (uint16_t)((x - 1) * DIM + y) : 0;
    uint16_t ka = (y > 0) ? (uint16_t)(x * DIM + y - 1) : 0;
    uint16_t kb = (y < DIM - 1) ? (uint16_t)(x * DIM + y + 1) : 0;
    real a = (real)0.5f * (im[kr] - im[kl]);
    real b = (real)0.5f * (im[kb] - im[ka]);
#ifdef TDI_REAL_DOUBLE
    real hh = 1e-16 + RSQRT((4 * a) * a + (4 * b) * b);
#else
    real hh = 1e-16f + RSQRT((4 * a) * a + (4 * b) * b);
#endif
    *gx = a; *gy = b; *h = hh;
    *gxn = ((real)2 * a) / hh;
    *gyn = ((real)2 * b) / hh;
}

/* Render of one frame from its fragments (renderer.cu:635-730 or :737-791): shade, paint
 * the owners into a zero image (fill_tex_im1, funcs.cu:800-817), blur, gradients at every
 * fragment (render and blurred target), correlation sum. g = [8][N]:
 * gx, gy, h, gxn, gyn (render) and gxsn, gysn (target), spare. */
enum { G_GX = 0, G_GY, G_H, G_GXN, G_GYN, G_GXSN, G_GYSN, G_N };

static double render_from_frags(const o_model *m, const o_frags *fr, const real *geo,
                                const real *R, const real *tau, const real *lam, real Lint,
                                const real *target_blurred, const float *taps,
                                real *sh, real *g, real *img, real *tmp, real *imb)
{
    const int N = fr->n;
    shade(m, geo, fr, R, tau, lam, Lint, sh, N);
    for (int p = 0; p < NPIX; ++p) img[p] = 0;
    for (int n = 0; n < N; ++n)
        if (fr->owner[n]) img[fr->pix[n]] = sh[SH_TEX * N + n];
    blur(taps, img, tmp, imb);
    double corr = 0.0;
    for (int n = 0; n < N; ++n) {
        real gx, gy, gxn, gyn, h, sgx, sgy, sgxn, sgyn, sh_;
        pixel_grad(imb, fr->pix[n], &gx, &gy, &gxn, &gyn, &h);
        pixel_grad(target_blurred, fr->pix[n], &sgx, &sgy, &sgxn, &sgyn, &sh_);
        g[G_GX * N + n] = gx; g[G_GY * N + n] = gy; g[G_H * N + n] = h;
        g[G_GXN * N + n] = gxn; g[G_GYN * N + n] = gyn;
        g[G_GXSN * N + n] = sgxn; g[G_GYSN * N + n] = sgyn;
        corr += (double)gxn * (double)sgxn + (double)gyn * (double)sgyn;
    }
    return corr;
}

/* ------------------------------------------------------------------------------------ */
/* Neighbour maps: DerivativeComputer::compute_hessian_and_gradient (derivative_computer.cu:
 * 43-72) with fill_ks_and_M0, fill_ksides, fill_krels, fill_krels2 (funcs.cu:81-131,
 * 288-343). For each fragment n, the fragments whose image differences define the
 * horizontal (kr - kl) and vertical (kb - ka) derivative rows. nb = [4][N] as kl, kr, ka, kb. */

static int cmp_pix(const void *a, const void *b, void *ctx)
{
    const uint16_t *pix = (const uint16_t *)ctx;
    int ia = *(const int *)a, ib = *(const int *)b;
    if (pix[ia] != pix[ib]) return (int)pix[ia] - (int)pix[ib];
    return ia - ib;      /* thrust::sort_by_key on device keys is a stable radix sort */
}

static const uint16_t *g_sort_pix;
static int cmp_pix_g(const void *a, const void *b) { return cmp_pix(a, b, (void *)g_sort_pix); }

void o_neighbours(const uint16_t *pix, int N, int32_t *nb, uint32_t *flags)
{
    int *perm = (int *)malloc(sizeof(int) * N);    /* ks_sortidx: sorted pos -> fragment */
    int *inv = (int *)malloc(sizeof(int) * N);     /* ks_sortidx_sortidx: fragment -> sorted pos */
    int *cum = (int *)calloc(NPIX, sizeof(int));   /* inclusive scan of M0 */
    int32_t *S = (int32_t *)calloc(4 * (size_t)N, sizeof(int32_t));
    for (int n = 0; n < N; ++n) { perm[n] = n; cum[pix[n]] = 1; }
    for (int p = 1; p < NPIX; ++p) cum[p] += cum[p - 1];
    /* (the M0 marks are 0/1, so the scan above equals thrust::inclusive_scan(M0)) */
    #pragma omp critical(o_sort)
    {
        g_sort_pix = pix;
        qsort(perm, N, sizeof(int), cmp_pix_g);
    }
    for (int i = 0; i < N; ++i) inv[perm[i]] = i;
    for (int i = 1; i < N - 1; ++i) {
        const int p = pix[perm[i]];
        const int y = p % DIM, x = p / DIM;
        const int right = (x < DIM - 1) ? (x + 1) * DIM + y : 0;
        const int left = (x > 0) ? (x - 1) * DIM + y : 0;
        int dl = cum[p] - cum[left];
        int kl = (i > dl) ? (i - dl) : 0;
        kl = (uint16_t)kl;
        if (kl >= N - 1) kl = N - 1;
        int kr = (uint16_t)(i + cum[right] - cum[p]);
        S[0 * N + i] = kl;
        S[1 * N + i] = kr;
        S[2 * N + i] = (uint16_t)(i - 1);
        S[3 * N + i] = (uint16_t)(i + 1);
    }
    for (int n = 0; n < N; ++n) {
        const int i = inv[n];
        for (int q = 0; q < 4; ++q) {
            int s = S[q * N + i];
            if (s >= N) { *flags |= O_FLAG_OUT_OF_DOMAIN; s = 0; }
            nb[q * N + n] = perm[s];
        }
    }
    free(perm); free(inv); free(cum); free(S);
}

/* ------------------------------------------------------------------------------------ */
/* Jacobian rows dI/dtheta [N][K+6]: fill_optimization_auxiliary_variables_phase1
 * (newfuncs.cu:173-255) for pose, render_expression_basis_texture_colmajor_rotated2_via_object
 * (funcs.cu:224-282) + fill_optimization_dI_depsilon_userotated (newfuncs.cu:265-299)
 * for expressions. Column order: epsilon[K], tau_x, tau_y, tau_z, u1, u2, u3. */

static void jacobian_rows(const o_model *m, const o_frags *fr, const real *sh, const real *g,
                          const real *R, const real *dR, const float *cam, real *J)
{
    const int N = fr->n, K = m->K, T = m->T, KT = K + 6;
    const real phix = cam[0], phiy = cam[1];
    for (int n = 0; n < N; ++n) {
        const int tri = fr->tri[n];
        const int ib = m->tl[tri], ic = m->tl[T + tri], ia = m->tl[2 * T + tri];
        const real al = fr->al[n], be = fr->be[n], ga = fr->ga[n];
        const real px = sh[(SH_P + 0) * N + n], py = sh[(SH_P + 1) * N + n], pz = sh[(SH_P + 2) * N + n];
        const real vx = sh[(SH_V + 0) * N + n], vy = sh[(SH_V + 1) * N + n], vz = sh[(SH_V + 2) * N + n];
        const real ivz = sh[SH_IVZ * N + n], ivz2 = sh[SH_IVZ2 * N + n];
        const real gx = g[G_GX * N + n], gy = g[G_GY * N + n];
        real *row = J + (size_t)n * KT;
        for (int k = 0; k < K; ++k) {
            const float *eb = m->E + (size_t)ib * 3 * K, *ec = m->E + (size_t)ic * 3 * K, *ea = m->E + (size_t)ia * 3 * K;
            real tx = ((real)eb[k] * al + (real)ec[k] * be) + (real)ea[k] * ga;
            real ty = ((real)eb[K + k] * al + (real)ec[K + k] * be) + (real)ea[K + k] * ga;
            real tz = ((real)eb[2 * K + k] * al + (real)ec[2 * K + k] * be) + (real)ea[2 * K + k] * ga;
            real REX = (tx * R[0] + ty * R[3]) + tz * R[6];
            real REY = (tx * R[1] + ty * R[4]) + tz * R[7];
            real REZ = (tx * R[2] + ty * R[5]) + tz * R[8];
            real nwx = (phix * ivz2) * (REX * vz - REZ * vx);
            real nwy = (phiy * ivz2) * (REY * vz - REZ * vy);
            row[k] = -(gx * nwx + gy * nwy);
        }
        real dWx_tx = phix * ivz, dWx_ty = 0, dWx_tz = ((-phix) * vx) * ivz2;
        real dWy_tx = 0, dWy_ty = phiy * ivz, dWy_tz = ((-phiy) * vy) * ivz2;
        row[K + 0] = -(gx * dWx_tx + gy * dWy_tx);
        row[K + 1] = -(gx * dWx_ty + gy * dWy_ty);
        row[K + 2] = -(gx * dWx_tz + gy * dWy_tz);
        for (int a = 0; a < 3; ++a) {
            const real *d = dR + 9 * a;
            real dvx = (d[0] * px + d[3] * py) + d[6] * pz;
            real dvy = (d[1] * px + d[4] * py) + d[7] * pz;
            real dvz = (d[2] * px + d[5] * py) + d[8] * pz;
            real dWx = (phix * ivz2) * (vz * dvx - vx * dvz);
            real dWy = (phiy * ivz2) * (vz * dvy - vy * dvz);
            row[K + 3 + a] = -(gx * dWx + gy * dWy);
        }
    }
}

/* Chain rule through the normalised gradient: fill_optimization_auxiliary_variables_phase2_new
 * (newfuncs.cu:417-463). Returns the two rows d(gx/|g|)/dtheta, d(gy/|g|)/dtheta of one
 * fragment from the rows of its four neighbours. */
static inline void chain_rows(const real *J, int ncols, int ld, const int32_t *nb, int N, int n,
                              const real *g, real *gxrow, real *gyrow)
{
    const real *Jr = J + (size_t)nb[1 * N + n] * ld, *Jl = J + (size_t)nb[0 * N + n] * ld;
    const real *Jb = J + (size_t)nb[3 * N + n] * ld, *Ja = J + (size_t)nb[2 * N + n] * ld;
    const real gx = g[G_GX * N + n], gy = g[G_GY * N + n], h = g[G_H * N + n];
    const real diffx = 2 * gx, diffy = 2 * gy;
    const real pre = (real)(1.0 / (0.001 + (double)(h * h * h)));
    for (int j = 0; j < ncols; ++j) {
        real dh = Jr[j] - Jl[j];
        real dv = Jb[j] - Ja[j];
        real X = (-diffy) * (-dh) - (-diffx) * (-dv);
        gxrow[j] = ((-pre) * (-diffy)) * X;
        gyrow[j] = (pre * (-diffx)) * X;
    }
}

/* ------------------------------------------------------------------------------------ */
/* Log-barrier terms of the image fit: Logbarrier_Initializer::compute_gradient_and_hessian
 * (logbarrier_initializer.cu:1272-1843) with compute_Gs (:456-520),
 * fill_optimization_dc_landmark (:587-697), fill_optimization_dI_depsilon_landmark
 * (:836-912), update_gradient (:915-929), update_diagonal_of_hessian_wbounds (:932-949),
 * and evaluate_objective_function (:1921-2093). No slack, no identity, no smoothing
 * (the video fit's configuration, video_fitter.cu:16-38). Hb [KT][KT] column-major and gb
 * are added to (not overwritten); returns the barrier objective (NaN when infeasible). */

static double barrier(const o_model *m, const o_frame *f, const real *x, const real *R,
                      const real *dR, int finetune_bounds, real *Hb, real *gb)
{
    const int K = m->K, KT = K + 6, V = m->V;
    const real *tau = x + K;
    const float *lb = finetune_bounds ? m->eps_lb_ft : m->eps_lb;
    const float *ub = finetune_bounds ? m->eps_ub_ft : m->eps_ub;
    const real phix = f->phix, phiy = f->phiy, cx = f->cx, cy = f->cy;
    const real fs = f->face_size;
    real p[NL * 3], Rp[NL * 3], G[4][NL];
    for (int i = 0; i < NL; ++i) {
        const int v = m->lis[i];
        for (int c = 0; c < 3; ++c) {
            const float *e = m->E + ((size_t)v * 3 + c) * K;
            real acc = 0;
            for (int k = 0; k < K; ++k) acc = RFMA((real)e[k], x[k], acc);
            p[i * 3 + c] = (real)m->mean[c * V + v] + acc;
        }
        for (int r = 0; r < 3; ++r)
            Rp[i * 3 + r] = (R[r] * p[i * 3] + R[r + 3] * p[i * 3 + 1]) + R[r + 6] * p[i * 3 + 2];
    }
    double obj = 0.0;
    for (int k = 0; k < K; ++k) {
        real fub = x[k] - (real)ub[k];
        real flb = (real)lb[k] - x[k];
        obj += (double)(-RLOG(-flb));
        obj += (double)(-RLOG(-fub));
    }
    for (int i = 0; i < NL; ++i) {
        const real r1p = Rp[i * 3], r2p = Rp[i * 3 + 1], r3p = Rp[i * 3 + 2];
        const real xproj = phix * ((r1p + tau[0]) / (r3p + tau[2])) + cx;
        const real yproj = phiy * ((r2p + tau[1]) / (r3p + tau[2])) + cy;
        const real xl = f->xl[i], yl = f->yl[i];
        G[0][i] = (real)0 - ((xl + (real)f->bounds[0 * NL + i] * fs) - xproj);
        G[1][i] = (real)0 - ((yl + (real)f->bounds[1 * NL + i] * fs) - yproj);
        G[2][i] = (real)0 - ((xproj - (real)f->bounds[2 * NL + i] * fs) - xl);
        G[3][i] = (real)0 - ((yproj - (real)f->bounds[3 * NL + i] * fs) - yl);
    }
    for (int s = 0; s < 4; ++s)
        for (int i = 0; i < NL; ++i) obj += (double)(-RLOG(G[s][i]));
    if (!Hb) return obj;

    /* for_nablaPhi_{Gx-,Gy-,Gx+,Gy+}: [4][NL][KT] */
    real *F = (real *)calloc(4 * (size_t)NL * KT, sizeof(real));
    for (int i = 0; i < NL; ++i) {
        const real px = p[i * 3], py = p[i * 3 + 1], pz = p[i * 3 + 2];
        const real vx = Rp[i * 3] + tau[0], vy = Rp[i * 3 + 1] + tau[1], vz = Rp[i * 3 + 2] + tau[2];
        const real ivz = (real)1 / vz, ivz2 = ivz * ivz;
        real nWx[16], nWy[16];
        nWx[0] = phix * ivz; nWx[1] = 0; nWx[2] = ((-phix) * vx) * ivz2;
        nWy[0] = 0; nWy[1] = phiy * ivz; nWy[2] = ((-phiy) * vy) * ivz2;
        for (int a = 0; a < 3; ++a) {
            const real *d = dR + 9 * a;
            real dvx = (d[0] * px + d[3] * py) + d[6] * pz;
            real dvy = (d[1] * px + d[4] * py) + d[7] * pz;
            real dvz = (d[2] * px + d[5] * py) + d[8] * pz;
            nWx[3 + a] = (phix * ivz2) * (vz * dvx - vx * dvz);
            nWy[3 + a] = (phiy * ivz2) * (vz * dvy - vy * dvz);
        }
        for (int c = 0; c < 6; ++c) {
            F[(0 * NL + i) * KT + K + c] = -nWx[c] / G[0][i];
            F[(1 * NL + i) * KT + K + c] = -nWy[c] / G[1][i];
            F[(2 * NL + i) * KT + K + c] = nWx[c] / G[2][i];
            F[(3 * NL + i) * KT + K + c] = nWy[c] / G[3][i];
        }
        const int v = m->lis[i];
        const float *ex = m->E + (size_t)v * 3 * K;
        for (int k = 0; k < K; ++k) {
            real RIX = ex[k], RIY = ex[K + k], RIZ = ex[2 * K + k];
            real dvx = (RIX * R[0] + RIY * R[3]) + RIZ * R[6];
            real dvy = (RIX * R[1] + RIY * R[4]) + RIZ * R[7];
            real dvz = (RIX * R[2] + RIY * R[5]) + RIZ * R[8];
            real wx = (phix * ivz2) * (dvx * vz - dvz * vx);
            real wy = (phiy * ivz2) * (dvy * vz - dvz * vy);
            F[(0 * NL + i) * KT + k] = -wx / G[0][i];
            F[(1 * NL + i) * KT + k] = -wy / G[1][i];
            F[(2 * NL + i) * KT + k] = wx / G[2][i];
            F[(3 * NL + i) * KT + k] = wy / G[3][i];
        }
    }
    for (int a = 0; a < KT; ++a) {
        double gs = 0.0;
        for (int i = 0; i < NL; ++i)
            for (int s = 0; s < 4; ++s) gs += (double)F[(s * NL + i) * KT + a];
        real ga = (real)gs;
        if (a < K) {
            real fub = x[a] - (real)ub[a];
            real flb = (real)lb[a] - x[a];
            ga = ga + ((real)-1 / fub + (real)1 / flb);
        }
        gb[a] += ga;
        for (int b = 0; b <= a; ++b) {
            double hs = 0.0;
            for (int s = 0; s < 4; ++s)
                for (int i = 0; i < NL; ++i)
                    hs += (double)F[(s * NL + i) * KT + a] * (double)F[(s * NL + i) * KT + b];
            real hv = (real)hs;
            if (a == b && a < K) {
                real fub = x[a] - (real)ub[a];
                real flb = (real)lb[a] - x[a];
                real nu = (real)(-1.0 / ((double)fub + 1e-12));
                real nl = (real)(1.0 / ((double)flb + 1e-12));
                hv = hv + (nu * nu + nl * nl);
            }
            Hb[(size_t)a * KT + b] += hv;
            if (a != b) Hb[(size_t)b * KT + a] += hv;
        }
    }
    free(F);
    return obj;
}

/* ------------------------------------------------------------------------------------ */
/* Solver::solve (solver.h:70-105): FP64 Cholesky of H (lower triangle), x = H^-1 g,
 * direction d = -x. Returns 0 and NaN directions when the factorisation fails. */
static int solve(const real *H, const real *g, int n, real *d, float damping)
{
    double *L = (double *)malloc(sizeof(double) * n * n);
    double *y = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n * n; ++i) L[i] = (double)H[i];
    /* damped solve (H + lambda I) x = g, lambda added in double; 0 = the reference's solve */
    for (int i = 0; i < n; ++i) L[i * n + i] += (double)damping;
    int ok = 1;
    for (int j = 0; j < n && ok; ++j) {
        double s = L[j * n + j];
        for (int k = 0; k < j; ++k) s -= L[k * n + j] * L[k * n + j];
        if (!(s > 0.0)) { ok = 0; break; }
        double ljj = sqrt(s);
        L[j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            double t = L[j * n + i];
            for (int k = 0; k < j; ++k) t -= L[k * n + i] * L[k * n + j];
            L[j * n + i] = t / ljj;
        }
    }
    if (ok) {
        for (int i = 0; i < n; ++i) {
            double t = (double)g[i];
            for (int k = 0; k < i; ++k) t -= L[k * n + i] * y[k];
            y[i] = t / L[i * n + i];
        }
        /* back substitution: the terms of row i are subtracted in decreasing k (the order in
         * which the y_k become known; cuSOLVER's DPOTRS order in the reference is the
         * library's) */
        for (int i = n - 1; i >= 0; --i) {
            double t = y[i];
            for (int k = n - 1; k > i; --k) t -= L[i * n + k] * y[k];
            y[i] = t / L[i * n + i];
        }
        for (int i = 0; i < n; ++i) d[i] = (real)(-y[i]);
    } else {
        for (int i = 0; i < n; ++i) d[i] = (real)NAN;
    }
    free(L); free(y);
    return ok;
}

/* The shape fit's solve (Solver::solve, solver.h:70-105, for the image fit's K+6 unknowns)
 * with reciprocal pivots: r_j = 1 / l_jj once per column, L(i,j) = t_ij * r_j; forward
 * y_i = (g_i - sum_k L(i,k) y_k) * r_i (terms in increasing k); back x_i = (y_i -
 * sum_k L(k,i) x_k) * r_i (terms in decreasing k); d = -x. The dot products are those of
 * solve(); the reference's cuSOLVER order is the library's. */
static int solve_shape(const real *H, const real *g, int n, real *d, float damping)
{
    double *L = (double *)malloc(sizeof(double) * n * n);
    double *y = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n * n; ++i) L[i] = (double)H[i];
    for (int i = 0; i < n; ++i) L[i * n + i] += (double)damping;
    int ok = 1;
    for (int j = 0; j < n && ok; ++j) {
        double s = L[j * n + j];
        for (int k = 0; k < j; ++k) s -= L[k * n + j] * L[k * n + j];
        if (!(s > 0.0)) { ok = 0; break; }
        const double ljj = sqrt(s);
        L[j * n + j] = ljj;
        r[j] = 1.0 / ljj;
        for (int i = j + 1; i < n; ++i) {
            double t = L[j * n + i];
            for (int k = 0; k < j; ++k) t -= L[k * n + i] * L[k * n + j];
            L[j * n + i] = t * r[j];
        }
    }
    if (ok) {
        for (int i = 0; i < n; ++i) {
            double t = (double)g[i];
            for (int k = 0; k < i; ++k) t -= L[k * n + i] * y[k];
            y[i] = t * r[i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double t = y[i];
            for (int k = n - 1; k > i; --k) t -= L[i * n + k] * y[k];
            y[i] = t * r[i];
        }
        for (int i = 0; i < n; ++i) d[i] = (real)(-y[i]);
    } else {
        for (int i = 0; i < n; ++i) d[i] = (real)NAN;
    }
    free(L); free(y); free(r);
    return ok;
}

/* ------------------------------------------------------------------------------------ */
/* Per-frame fitting context */

typedef struct {
    const o_model *m;
    const o_frame *f;
    const o_config *cfg;
    real *tgt;           /* blurred target */
    real *geo;           /* [8][V] */
    real *geo_f32src;    /* unused in FP32 */
    float *xpf, *ypf, *Zf;
    o_frags fr;
    int cap;
    real *sh, *g, *img, *tmp, *imb;
    real *J;             /* [N][KT] */
    int32_t *nb;
    real R[9], dR[27];
    o_report *rep;
} ctx_t;

static void ctx_init(ctx_t *c, const o_model *m, const o_frame *f, const o_config *cfg, o_report *rep)
{
    memset(c, 0, sizeof(*c));
    c->m = m; c->f = f; c->cfg = cfg; c->rep = rep;
    const int V = m->V;
    c->cap = 4 * m->T;
    c->tgt = (real *)malloc(sizeof(real) * NPIX);
    c->geo = (real *)malloc(sizeof(real) * 8 * V);
    c->xpf = (float *)malloc(sizeof(float) * V);
    c->ypf = (float *)malloc(sizeof(float) * V);
    c->Zf = (float *)malloc(sizeof(float) * V);
    c->fr.slot = (int32_t *)malloc(sizeof(int32_t) * c->cap);
    c->fr.tri = (int32_t *)malloc(sizeof(int32_t) * c->cap);
    c->fr.pix = (uint16_t *)malloc(sizeof(uint16_t) * c->cap);
    c->fr.al = (float *)malloc(sizeof(float) * c->cap);
    c->fr.be = (float *)malloc(sizeof(float) * c->cap);
    c->fr.ga = (float *)malloc(sizeof(float) * c->cap);
    c->fr.owner = (uint8_t *)malloc(c->cap);
    c->img = (real *)malloc(sizeof(real) * NPIX);
    c->tmp = (real *)malloc(sizeof(real) * NPIX);
    c->imb = (real *)malloc(sizeof(real) * NPIX);
    c->sh = NULL; c->g = NULL; c->J = NULL; c->nb = NULL;
    real *src = (real *)malloc(sizeof(real) * NPIX);
    for (int p = 0; p < NPIX; ++p) src[p] = f->target[p];
    blur(cfg->taps, src, c->tmp, c->tgt);
    free(src);
}

static void ctx_free(ctx_t *c)
{
    free(c->tgt); free(c->geo); free(c->xpf); free(c->ypf); free(c->Zf);
    free(c->fr.slot); free(c->fr.tri); free(c->fr.pix); free(c->fr.al); free(c->fr.be);
    free(c->fr.ga); free(c->fr.owner); free(c->img); free(c->tmp); free(c->imb);
    free(c->sh); free(c->g); free(c->J); free(c->nb);
}

static void ensure_frag_buffers(ctx_t *c)
{
    const int N = c->fr.n, KT = c->m->K + 6;
    free(c->sh); free(c->g); free(c->J); free(c->nb);
    c->sh = (real *)malloc(sizeof(real) * SH_N * (size_t)(N > 0 ? N : 1));
    c->g = (real *)malloc(sizeof(real) * G_N * (size_t)(N > 0 ? N : 1));
    c->J = (real *)malloc(sizeof(real) * (size_t)KT * (N > 0 ? N : 1));
    c->nb = (int32_t *)malloc(sizeof(int32_t) * 4 * (size_t)(N > 0 ? N : 1));
}

/* Geometry at x (vertex stage); returns the face-size check. */
static int geometry(ctx_t *c, const real *x, int with_deriv)
{
    const o_model *m = c->m;
    const int K = m->K, V = m->V;
    float cam[4] = {c->f->phix, c->f->phiy, c->f->cx, c->f->cy};
    o_rotation(x + K + 3, c->R, with_deriv ? c->dR : NULL);
    int ok = o_vertex_stage(m, x, c->R, x + K, cam, c->cfg->ref_face_size, c->geo);
    for (int v = 0; v < V; ++v) {
        c->xpf[v] = (float)c->geo[6 * V + v];
        c->ypf[v] = (float)c->geo[7 * V + v];
        c->Zf[v] = (float)c->geo[5 * V + v];
    }
    return ok;
}

/* Visibility of the current geometry. */
static void raster_frame(ctx_t *c)
{
    uint32_t fl = 0;
    o_raster(c->m, c->xpf, c->ypf, c->Zf, c->f->x0, c->f->y0, &c->fr, &fl);
    c->rep->flags |= fl;
    c->rep->renders++;
    ensure_frag_buffers(c);
    c->rep->n_fragments = c->fr.n;
}

static int geometry_and_raster(ctx_t *c, const real *x, int with_deriv)
{
    int ok = geometry(c, x, with_deriv);
    raster_frame(c);
    return ok;
}

/* Full image-term evaluation at x (render + optional Jacobian). Returns the correlation
 * sum (not scaled by tau). */
static double image_term(ctx_t *c, const real *x, const real *lam, real Lint)
{
    return render_from_frags(c->m, &c->fr, c->geo, c->R, x + c->m->K, lam, Lint, c->tgt,
                             c->cfg->taps, c->sh, c->g, c->img, c->tmp, c->imb);
}

/* Normal equations of the image term (derivative_computer.cu:135-164):
 * H = tau (Gx^T Gx + Gy^T Gy), g = -tau (gxs^T Gx + gys^T Gy). */
static void image_normal_equations(ctx_t *c, real tau, real *H, real *gvec)
{
    const o_model *m = c->m;
    const int N = c->fr.n, K = m->K, KT = K + 6;
    float cam[4] = {c->f->phix, c->f->phiy, c->f->cx, c->f->cy};
    uint32_t fl = 0;
    o_neighbours(c->fr.pix, N, c->nb, &fl);
    c->rep->flags |= fl;
    jacobian_rows(m, &c->fr, c->sh, c->g, c->R, c->dR, cam, c->J);
    /* The reference forms H and g with cublasSgemm (derivative_computer.cu:157-163), whose
     * summation order is the library's. The order here is fixed: fragments in chunks of
     * NE_CHUNK; within a chunk, from zero, one fused multiply-add per row and entry in fragment
     * order (x row, then y row); the chunk sums are then added in chunk order. In the FP32
     * build the rows are floats, so every product is exact in double and only the additions
     * round. */
    enum { NE_CHUNK = 256 };
    double *Hs = (double *)calloc((size_t)KT * KT, sizeof(double));
    double *gs = (double *)calloc(KT, sizeof(double));
    double *Hc = (double *)malloc(sizeof(double) * (size_t)KT * KT);
    double *gc = (double *)malloc(sizeof(double) * KT);
    real *gxr = (real *)malloc(sizeof(real) * KT), *gyr = (real *)malloc(sizeof(real) * KT);
    for (int c0 = 0; c0 < N; c0 += NE_CHUNK) {
        const int c1 = c0 + NE_CHUNK < N ? c0 + NE_CHUNK : N;
        memset(Hc, 0, sizeof(double) * (size_t)KT * KT);
        memset(gc, 0, sizeof(double) * KT);
        for (int n = c0; n < c1; ++n) {
            chain_rows(c->J, KT, KT, c->nb, N, n, c->g, gxr, gyr);
            const double sx = c->g[G_GXSN * N + n], sy = c->g[G_GYSN * N + n];
            for (int a = 0; a < KT; ++a) {
                const double xa = gxr[a], ya = gyr[a];
                gc[a] = fma(sy, ya, fma(sx, xa, gc[a]));
                double *hr = Hc + (size_t)a * KT;
                for (int b = 0; b <= a; ++b) hr[b] = fma(ya, (double)gyr[b], fma(xa, (double)gxr[b], hr[b]));
            }
        }
        for (int a = 0; a < KT; ++a) {
            gs[a] += gc[a];
            for (int b = 0; b <= a; ++b) Hs[(size_t)a * KT + b] += Hc[(size_t)a * KT + b];
        }
    }
    free(Hc); free(gc);
    for (int a = 0; a < KT; ++a) {
        gvec[a] = (real)(-(double)tau * gs[a]);
        for (int b = 0; b <= a; ++b) {
            real v = (real)((double)tau * Hs[(size_t)a * KT + b]);
            H[(size_t)a * KT + b] = v;
            H[(size_t)b * KT + a] = v;
        }
    }
    free(Hs); free(gs); free(gxr); free(gyr);
}

/* ------------------------------------------------------------------------------------ */
/* fit_3DMM_lambdas (model_fitter.cu:981-1073) with render_for_illumination_only
 * (renderer.cu:737-791) and compute_hessian_and_gradient_for_lambda
 * (derivative_computer.cu:235-312). Geometry is rendered once at x; only the light moves. */

static double illum_objective(ctx_t *c, const real *x, const real *lam, real Lint)
{
    return -image_term(c, x, lam, Lint);     /* grad_corr with alpha = 1 */
}

static void fit_lambdas(ctx_t *c, const real *x, real *lam, real Lint)
{
    const int N0 = 0; (void)N0;
    geometry_and_raster(c, x, 1);
    const int N = c->fr.n;
    if (c->rep->flags & O_FLAG_RENDER_SKIPPED) return;
    uint32_t fl = 0;
    o_neighbours(c->fr.pix, N, c->nb, &fl);
    c->rep->flags |= fl;
    real lam_ls[3];
    int terminate = 0;
    real *Jl = (real *)malloc(sizeof(real) * 3 * (size_t)(N > 0 ? N : 1));
    for (int it = 0; it < c->cfg->max_iters_lambda; ++it) {
        if (terminate) break;
        c->rep->iters_lambda++;
        real obj = (real)illum_objective(c, x, lam, Lint);
        for (int n = 0; n < N; ++n)
            for (int j = 0; j < 3; ++j) {
                real r0 = c->sh[(SH_DLAM + 0) * N + n], r1 = c->sh[(SH_DLAM + 1) * N + n], r2 = c->sh[(SH_DLAM + 2) * N + n];
                Jl[(size_t)n * 3 + j] = (r0 * c->R[j] + r1 * c->R[j + 3]) + r2 * c->R[j + 6];
            }
        double Hs[9] = {0}, gs[3] = {0};
        for (int n = 0; n < N; ++n) {
            real gxr[3], gyr[3];
            chain_rows(Jl, 3, 3, c->nb, N, n, c->g, gxr, gyr);
            const double sx = c->g[G_GXSN * N + n], sy = c->g[G_GYSN * N + n];
            for (int a = 0; a < 3; ++a) {
                gs[a] += sx * gxr[a] + sy * gyr[a];
                for (int b = 0; b < 3; ++b) Hs[a * 3 + b] += (double)gxr[a] * gxr[b] + (double)gyr[a] * gyr[b];
            }
        }
        real H[9], gv[3], d[3];
        for (int i = 0; i < 9; ++i) H[i] = (real)Hs[i];
        for (int i = 0; i < 3; ++i) gv[i] = (real)(-gs[i]);
        solve(H, gv, 3, d, 0.0f);
        {
            real l2n = (real)((double)d[0] * gv[0] + (double)d[1] * gv[1] + (double)d[2] * gv[2]);
            if (isnan((double)l2n)) break;    /* every trial would be rejected down to t < 0.01 */
        }
        real t = 1.0f;
        const real ALPHA = 0.5f, BETA = 0.5f;
        for (int inner = 0; inner < 1000;) {
            if (t < (real)0.01f) { terminate = 1; break; }
            for (int j = 0; j < 3; ++j) lam_ls[j] = lam[j] + t * d[j];
            real obj_tmp = (real)illum_objective(c, x, lam_ls, Lint);
            inner++;
            real l2 = (real)((double)d[0] * gv[0] + (double)d[1] * gv[1] + (double)d[2] * gv[2]);
            if ((double)(-l2) < 0.0003) { terminate = 1; break; }
            l2 = l2 * (ALPHA * t);
            if (obj_tmp < obj + l2) { for (int j = 0; j < 3; ++j) lam[j] = lam_ls[j]; break; }
            t = t * BETA;
        }
    }
    free(Jl);
}

/* ------------------------------------------------------------------------------------ */
/* fit_3DMM_shape_rigid (model_fitter.cu:121-375) and fit_3DMM_epsilon_finetune (:397-672),
 * with get_obj_hessian_and_gradient_multiframe (:21-116) for one frame. n_upd is the
 * number of leading entries a trial updates (all K+6, or the K expressions in the
 * finetune). x_ls persists across stages like ov_linesearch does in the reference. */

static int fit_shape(ctx_t *c, real *x, real *x_ls, const real *lam, real Lint, int finetune,
                     int max_iters, int32_t *iters_out)
{
    const o_model *m = c->m;
    const int K = m->K, KT = K + 6;
    const int n_upd = finetune ? KT - 6 : KT;
    const real tau_img = (real)5.0f * (real)5.0f;
    const real tthr = (real)0.075f;
    real *H = (real *)calloc((size_t)KT * KT, sizeof(real));
    real *gv = (real *)calloc(KT, sizeof(real));
    real *d = (real *)malloc(sizeof(real) * KT);
    int num_outer = 0, terminate = 0;
    for (int i = 0; i < max_iters; ++i) {
        num_outer++;
        if (terminate) break;
        /* full evaluation at x */
        geometry_and_raster(c, x, 1);
        if (c->rep->flags & O_FLAG_RENDER_SKIPPED) break;     /* the frame stops here */
        double corr = image_term(c, x, lam, Lint);
        real grad_corr = tau_img * (real)corr;
        image_normal_equations(c, tau_img, H, gv);
        double ob = barrier(m, c->f, x, c->R, c->dR, finetune, H, gv);
        grad_corr = grad_corr + (-(real)ob);
        if (!solve_shape(H, gv, KT, d, c->cfg->damping)) c->rep->flags |= O_FLAG_CHOL_FAILED;
        if (isnan((double)d[0])) { c->rep->flags |= O_FLAG_NAN_DIRECTION; terminate = 1; break; }
        real t = 1.0f;
        const real ALPHA = 0.4f, BETA = 0.8f;
        real obj = -grad_corr;
        c->rep->objective = (float)obj;
        double dg = 0.0;
        for (int a = 0; a < KT; ++a) dg += (double)d[a] * (double)gv[a];
        real l2base = (real)dg;
        for (int inner = 0; inner < 100;) {
            if (t < tthr) { terminate = 1; break; }
            for (int a = 0; a < n_upd; ++a) x_ls[a] = x[a] + t * d[a];
            if (x_ls[K + 2] < 0) {           /* stuck: every later outer iteration repeats */
                c->rep->flags |= O_FLAG_STUCK_NEG_TZ;
                terminate = 1; num_outer = max_iters; break;
            }
            int face_ok = geometry(c, x_ls, 0);
            if (!face_ok) { t = t * BETA; continue; }
            double obi = barrier(m, c->f, x_ls, c->R, NULL, finetune, NULL, NULL);
            if (isnan(obi)) { t = t * BETA; continue; }
            /* the -g.d test (model_fitter.cu:338-342) does not depend on the trial's render */
            if ((double)(-l2base) < 0.0003) { terminate = 1; break; }
            raster_frame(c);
            if (c->rep->flags & O_FLAG_RENDER_SKIPPED) { terminate = 2; break; }
            double corr_t = image_term(c, x_ls, lam, Lint);
            real gc = tau_img * (real)corr_t;
            gc = gc + (-(real)obi);
            real obj_tmp = -gc;
            inner++;
            real l2 = l2base;
            l2 = l2 * (ALPHA * t);
            if (obj_tmp < obj + l2) {
                for (int a = 0; a < KT; ++a) x[a] = x_ls[a];
                c->rep->objective = (float)obj_tmp;
                break;
            }
            t = t * BETA;
        }
        if (terminate == 2) break;
    }
    if (num_outer > max_iters) num_outer = max_iters;
    *iters_out += num_outer;
    free(H); free(gv); free(d);
    return num_outer > c->cfg->niters_success;
}

/* VideoFitter::fit_to_video_frame (video_fitter.cu:432-648) after the landmark
 * initialisation: target blur, light fit, shape fit(s), optional finetune. */
static void fit_frame(const o_model *m, const o_frame *f, const o_config *cfg, real *x,
                      real *lam, real Lint, o_report *rep)
{
    ctx_t c;
    memset(rep, 0, sizeof(*rep));
    ctx_init(&c, m, f, cfg, rep);
    const int KT = m->K + 6;
    real *x_ls = (real *)malloc(sizeof(real) * KT);
    memcpy(x_ls, x, sizeof(real) * KT);
    int ok = 0;
#define ALIVE (!(rep->flags & O_FLAG_RENDER_SKIPPED))
    fit_lambdas(&c, x, lam, Lint);
    if (ALIVE) {
        memcpy(x_ls, x, sizeof(real) * KT);
        ok = fit_shape(&c, x, x_ls, lam, Lint, 0, cfg->max_iters_rigid, &rep->iters_rigid);
    }
    if (cfg->twostage_illum) {
        for (int s = 0; s < 2 && ALIVE; ++s) {
            fit_lambdas(&c, x, lam, Lint);
            if (!ALIVE) break;
            memcpy(x_ls, x, sizeof(real) * KT);
            ok = fit_shape(&c, x, x_ls, lam, Lint, 0, cfg->max_iters_rigid, &rep->iters_rigid);
        }
    }
    if (cfg->finetune && ALIVE)
        fit_shape(&c, x, x_ls, lam, Lint, 1, cfg->max_iters_finetune, &rep->iters_finetune);
#undef ALIVE
    if (!ok || (rep->flags & O_FLAG_RENDER_SKIPPED)) rep->flags |= O_FLAG_FAIL;
    free(x_ls);
    ctx_free(&c);
}

/* ==================================================================================== */
/* Exported entry points (ctypes). States are float in memory in both builds. */

int o_fit_frames(const o_model *m, const o_frame *frames, int F, const o_config *cfg,
                 float *x /* [F][K+6] */, float *lam /* [F][3] */, const float *Lint /* [F] */,
                 o_report *rep, int n_threads)
{
    const int KT = m->K + 6;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < F; ++i) {
        real xr[512], lr[3];
        for (int a = 0; a < KT; ++a) xr[a] = x[(size_t)i * KT + a];
        for (int a = 0; a < 3; ++a) lr[a] = lam[i * 3 + a];
        fit_frame(m, &frames[i], cfg, xr, lr, (real)Lint[i], &rep[i]);
        for (int a = 0; a < KT; ++a) x[(size_t)i * KT + a] = (float)xr[a];
        for (int a = 0; a < 3; ++a) lam[i * 3 + a] = (float)lr[a];
    }
    return 0;
}

int o_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Rotation of one state, float in/out. */
void o_rotation_f(const float *u, float *R, float *dR)
{
    real ur[3] = {u[0], u[1], u[2]}, Rr[9], dRr[27];
    o_rotation(ur, Rr, dRr);
    for (int i = 0; i < 9; ++i) R[i] = (float)Rr[i];
    for (int i = 0; i < 27; ++i) dR[i] = (float)dRr[i];
}

/* Vertex stage of one state: geo [8][V] float. Returns the face check. */
int o_vertex_stage_f(const o_model *m, const float *x, const float *cam, float ref_face_size, float *geo)
{
    const int K = m->K, V = m->V;
    real *xr = (real *)malloc(sizeof(real) * (K + 6));
    real *g = (real *)malloc(sizeof(real) * 8 * V);
    for (int a = 0; a < K + 6; ++a) xr[a] = x[a];
    real R[9];
    o_rotation(xr + K + 3, R, NULL);
    int ok = o_vertex_stage(m, xr, R, xr + K, cam, ref_face_size, g);
    for (int i = 0; i < 8 * V; ++i) geo[i] = (float)g[i];
    free(xr); free(g);
    return ok;
}

/* Raster of given projections. Arrays sized 4*T. Returns N. */
int o_raster_f(const o_model *m, const float *xp, const float *yp, const float *Zc, int x0, int y0,
               int32_t *slot, int32_t *tri, uint16_t *pix, float *al, float *be, float *ga,
               uint8_t *owner, uint32_t *flags)
{
    o_frags fr = {0, slot, tri, pix, al, be, ga, owner};
    return o_raster(m, xp, yp, Zc, x0, y0, &fr, flags);
}

/* Neighbour maps of a fragment pixel list. */
void o_neighbours_f(const uint16_t *pix, int N, int32_t *nb, uint32_t *flags)
{
    o_neighbours(pix, N, nb, flags);
}

/* Blur of one image (float in/out). */
void o_blur_f(const float *taps, const float *src, float *dst)
{
    real *s = (real *)malloc(sizeof(real) * NPIX), *t = (real *)malloc(sizeof(real) * NPIX);
    real *d = (real *)malloc(sizeof(real) * NPIX);
    for (int p = 0; p < NPIX; ++p) s[p] = src[p];
    blur(taps, s, t, d);
    for (int p = 0; p < NPIX; ++p) dst[p] = (float)d[p];
    free(s); free(t); free(d);
}

/* One full evaluation at a state (what one outer GN iteration computes before the line
 * search), with every intermediate a parity test needs. Output buffers are optional
 * (NULL skips them); frag buffers sized 4*T.
 *   image      [65536]  blurred render
 *   sh         [14][cap] per-fragment shading (layout of the SH_* enum)
 *   grads      [8][cap]  gx, gy, h, gxn, gyn, gxsn, gysn
 *   nb         [4][cap]  kl, kr, ka, kb
 *   J          [cap][K+6] Jacobian rows
 *   H [KT*KT], g [KT]: image + barrier normal equations; d [KT] search direction
 *   scal[4]: correlation sum, barrier objective, objective (-grad_corr), face check */
int o_evaluate_f(const o_model *m, const o_frame *f, const o_config *cfg, const float *x,
                 const float *lam, float Lint, int finetune_bounds,
                 int32_t *slot, int32_t *tri, uint16_t *pix, float *al, float *be, float *ga, uint8_t *owner,
                 float *image, float *sh, float *grads, int32_t *nb, float *J,
                 float *H, float *g, float *d, double *scal, uint32_t *flags)
{
    o_report rep;
    memset(&rep, 0, sizeof(rep));
    ctx_t c;
    ctx_init(&c, m, f, cfg, &rep);
    const int K = m->K, KT = K + 6;
    real xr[512], lr[3] = {lam[0], lam[1], lam[2]};
    for (int a = 0; a < KT; ++a) xr[a] = x[a];
    int face_ok = geometry_and_raster(&c, xr, 1);
    const int N = c.fr.n;
    double corr = image_term(&c, xr, lr, (real)Lint);
    real *Hr = (real *)calloc((size_t)KT * KT, sizeof(real));
    real *gr = (real *)calloc(KT, sizeof(real));
    real *dr = (real *)calloc(KT, sizeof(real));
    const real tau_img = (real)25.0f;
    image_normal_equations(&c, tau_img, Hr, gr);
    double ob = barrier(m, f, xr, c.R, c.dR, finetune_bounds, Hr, gr);
    if (!solve_shape(Hr, gr, KT, dr, cfg->damping)) rep.flags |= O_FLAG_CHOL_FAILED;
    real grad_corr = tau_img * (real)corr;
    grad_corr = grad_corr + (-(real)ob);
    if (slot) memcpy(slot, c.fr.slot, sizeof(int32_t) * N);
    if (tri) memcpy(tri, c.fr.tri, sizeof(int32_t) * N);
    if (pix) memcpy(pix, c.fr.pix, sizeof(uint16_t) * N);
    if (al) memcpy(al, c.fr.al, sizeof(float) * N);
    if (be) memcpy(be, c.fr.be, sizeof(float) * N);
    if (ga) memcpy(ga, c.fr.ga, sizeof(float) * N);
    if (owner) memcpy(owner, c.fr.owner, N);
    if (image) for (int p = 0; p < NPIX; ++p) image[p] = (float)c.imb[p];
    if (sh) for (int q = 0; q < SH_N; ++q) for (int n = 0; n < N; ++n) sh[(size_t)q * N + n] = (float)c.sh[(size_t)q * N + n];
    if (grads) for (int q = 0; q < G_N; ++q) for (int n = 0; n < N; ++n) grads[(size_t)q * N + n] = (float)c.g[(size_t)q * N + n];
    if (nb) memcpy(nb, c.nb, sizeof(int32_t) * 4 * N);
    if (J) for (size_t i = 0; i < (size_t)N * KT; ++i) J[i] = (float)c.J[i];
    if (H) for (int i = 0; i < KT * KT; ++i) H[i] = (float)Hr[i];
    if (g) for (int i = 0; i < KT; ++i) g[i] = (float)gr[i];
    if (d) for (int i = 0; i < KT; ++i) d[i] = (float)dr[i];
    if (scal) { scal[0] = corr; scal[1] = ob; scal[2] = (double)(-grad_corr); scal[3] = face_ok; }
    if (flags) *flags = rep.flags;
    free(Hr); free(gr); free(dr);
    ctx_free(&c);
    return N;
}

/* The image term alone at a state: H = tau (Gx^T Gx + Gy^T Gy) and g = -tau (gxs^T Gx +
 * gys^T Gy) (derivative_computer.cu:135-164) without the barrier terms, and the correlation
 * sum; what the reference's DerivativeComputer forms before Logbarrier_Initializer adds its
 * part. Returns N. */
int o_image_terms_f(const o_model *m, const o_frame *f, const o_config *cfg, const float *x,
                    const float *lam, float Lint, float tau_img, float *H, float *g, double *corr)
{
    o_report rep;
    memset(&rep, 0, sizeof(rep));
    ctx_t c;
    ctx_init(&c, m, f, cfg, &rep);
    const int KT = m->K + 6;
    real xr[512], lr[3] = {lam[0], lam[1], lam[2]};
    for (int a = 0; a < KT; ++a) xr[a] = x[a];
    geometry_and_raster(&c, xr, 1);
    const int N = c.fr.n;
    double cs = image_term(&c, xr, lr, (real)Lint);
    const size_t nkt = (size_t)(KT > 0 ? KT : 1);
    real *Hr = (real *)calloc(nkt * nkt, sizeof(real));
    real *gr = (real *)calloc(nkt, sizeof(real));
    image_normal_equations(&c, (real)tau_img, Hr, gr);
    for (int i = 0; i < KT * KT; ++i) H[i] = (float)Hr[i];
    for (int i = 0; i < KT; ++i) g[i] = (float)gr[i];
    if (corr) *corr = cs;
    free(Hr); free(gr);
    ctx_free(&c);
    return N;
}

/* Render one state to an image without fitting (used to synthesise targets in tests). */
int o_render_image_f(const o_model *m, const o_frame *f, const o_config *cfg, const float *x,
                     const float *lam, float Lint, float *unblurred, uint32_t *flags)
{
    o_report rep;
    memset(&rep, 0, sizeof(rep));
    ctx_t c;
    ctx_init(&c, m, f, cfg, &rep);
    const int KT = m->K + 6;
    real xr[512], lr[3] = {lam[0], lam[1], lam[2]};
    for (int a = 0; a < KT; ++a) xr[a] = x[a];
    geometry_and_raster(&c, xr, 0);
    image_term(&c, xr, lr, (real)Lint);
    for (int p = 0; p < NPIX; ++p) unblurred[p] = (float)c.img[p];
    if (flags) *flags = rep.flags;
    int N = c.fr.n;
    ctx_free(&c);
    return N;
}

/* ------------------------------------------------------------------------------------ */
/* OrthographicInitializer::fit_model (orthographic_initializer.cu:243-380) for one frame:
 * a Gauss-Newton fit of x = (tau_x, tau_y, sigma_x, sigma_y, u1, u2, u3) so that the scaled
 * orthographic projection (sigma_x (R p + tau)_x, sigma_y (R p + tau)_y) of the model's
 * landmark points p (p0L, [3][51]) meets the centred landmarks, from the reference's start
 * point (0, 0, 15, 15, 0, 0, 0.05) (:152-167), Armijo line search with alpha 0.4 and beta 0.5
 * down to t = 0.1, at most 100 outer iterations. FP32 as the reference; its library calls in
 * a fixed order: landmark means as sequential float sums (thrust::reduce), R p as
 * ((R0 p0 + R3 p1) + R6 p2) (cublasSgemm), J^T J, J^T e and the dot products as float fused
 * multiply-add chains over the 102 residual rows in order (x rows, then y rows), the 7 x 7
 * system with solve(). Writes x and the rotation of the last trial point (the one the
 * reference's Euler angles are read from, :366-373). Returns the outer iterations run. */
#define ORTH_N 7
#define ORTH_ROWS (2 * O_NL)

static void orth_rp(const float *R, const float *p0L, int i, float *r)
{
    const float p0 = p0L[i], p1 = p0L[O_NL + i], p2 = p0L[2 * O_NL + i];
    for (int k = 0; k < 3; ++k) r[k] = (R[k] * p0 + R[3 + k] * p1) + R[6 + k] * p2;
}

/* The Gauss-Newton iterations of OrthographicInitializer::fit_model from the start point in x
 * (reset_variables = false continues from x, orthographic_initializer.cu:243-250). */
static int orth_fit(const float *xl, const float *yl, const float *p0L, float *x, float *R_last)
{
    float xb[O_NL], yb[O_NL], xm = 0.0f, ym = 0.0f;
    for (int i = 0; i < O_NL; ++i) { xm += xl[i]; ym += yl[i]; }
    xm = xm / (float)O_NL;
    ym = ym / (float)O_NL;
    for (int i = 0; i < O_NL; ++i) { xb[i] = xl[i] - xm; yb[i] = yl[i] - ym; }
    for (int k = 0; k < 9; ++k) R_last[k] = 0.0f;
    int terminate = 0, q;
    for (q = 0; q < 100; ++q) {
        if (terminate) break;
        float R[9], dR[27];
        o_rotation_f(x + 4, R, dR);
        float W[ORTH_N][ORTH_ROWS];
        float e[ORTH_ROWS];
        for (int i = 0; i < O_NL; ++i) {
            float rp[3], d[3][3];
            orth_rp(R, p0L, i, rp);
            for (int a = 0; a < 3; ++a) orth_rp(dR + 9 * a, p0L, i, d[a]);
            W[0][i] = x[2];        W[0][O_NL + i] = 0.0f;
            W[1][i] = 0.0f;        W[1][O_NL + i] = x[3];
            W[2][i] = x[0] + rp[0]; W[2][O_NL + i] = 0.0f;
            W[3][i] = 0.0f;        W[3][O_NL + i] = x[1] + rp[1];
            for (int a = 0; a < 3; ++a) {
                W[4 + a][i] = x[2] * d[a][0];
                W[4 + a][O_NL + i] = x[3] * d[a][1];
            }
            e[i] = x[2] * (rp[0] + x[0]) - xb[i];
            e[O_NL + i] = x[3] * (rp[1] + x[1]) - yb[i];
        }
        float JTJ[ORTH_N * ORTH_N], dg[ORTH_N], obj = 0.0f, sd[ORTH_N];
        for (int a = 0; a < ORTH_N; ++a)
            for (int b = 0; b < ORTH_N; ++b) {
                float s = 0.0f;
                for (int r = 0; r < ORTH_ROWS; ++r) s = fmaf(W[a][r], W[b][r], s);
                JTJ[b * ORTH_N + a] = s;
            }
        for (int a = 0; a < ORTH_N; ++a) {
            float s = 0.0f;
            for (int r = 0; r < ORTH_ROWS; ++r) s = fmaf(W[a][r], e[r], s);
            dg[a] = s;
        }
        for (int r = 0; r < ORTH_ROWS; ++r) obj = fmaf(e[r], e[r], obj);
        {
            real Hr[ORTH_N * ORTH_N], gr[ORTH_N], dr[ORTH_N];   /* exact copies in either build */
            for (int k = 0; k < ORTH_N * ORTH_N; ++k) Hr[k] = JTJ[k];
            for (int k = 0; k < ORTH_N; ++k) gr[k] = dg[k];
            solve(Hr, gr, ORTH_N, dr, 0.0f);
            for (int k = 0; k < ORTH_N; ++k) sd[k] = (float)dr[k];
        }
        float t = 1.0f;
        for (int inner = 0; inner < 1000; ++inner) {
            if (t < 0.1f) { terminate = 1; break; }
            float xs[ORTH_N], Rt[9], dRt[27];
            for (int n = 0; n < ORTH_N; ++n) xs[n] = x[n] + t * sd[n];
            o_rotation_f(xs + 4, Rt, dRt);
            for (int k = 0; k < 9; ++k) R_last[k] = Rt[k];
            float et[ORTH_ROWS], objt = 0.0f, tmp = 0.0f;
            for (int i = 0; i < O_NL; ++i) {
                float rp[3];
                orth_rp(Rt, p0L, i, rp);
                et[i] = xs[2] * (rp[0] + xs[0]) - xb[i];
                et[O_NL + i] = xs[3] * (rp[1] + xs[1]) - yb[i];
            }
            for (int r = 0; r < ORTH_ROWS; ++r) objt = fmaf(et[r], et[r], objt);
            for (int n = 0; n < ORTH_N; ++n) tmp = fmaf(sd[n], dg[n], tmp);
            tmp *= 0.4f * t;
            if (objt < obj + tmp) {
                for (int n = 0; n < ORTH_N; ++n) x[n] = xs[n];
                break;
            }
            t = t * 0.5f;
        }
    }
    return q;
}

int o_orthographic_f(const float *xl, const float *yl, const float *p0L, float *x, float *R_last)
{
    /* reset_orthographic (orthographic_initializer.cu:133-153): the reference's start point */
    const float x0[ORTH_N] = {0.0f, 0.0f, 15.0f, 15.0f, 0.0f, 0.0f, 0.05f};
    for (int n = 0; n < ORTH_N; ++n) x[n] = x0[n];
    return orth_fit(xl, yl, p0L, x, R_last);
}

/* ------------------------------------------------------------------------------------ */
/* Landmark initialisation of one frame, as VideoFitter::fit_to_video_frame runs it before the
 * image fit (video_fitter.cu:456-500): Logbarrier_Initializer::initialize_with_orthographic_t
 * (logbarrier_initializer.cu:1862-1918), set_minimal_slack (:1041-1092) and fit_model with a
 * slack variable (:1095-1269; compute_gradient_and_hessian :1272-1843, evaluate_objective_function
 * :1921-2093, compute_Gs :456-520, fill_optimization_dc_landmark :587-697,
 * fill_optimization_dI_depsilon_landmark :836-912, fill_for_nabla2F_dsdc :780-818). One frame,
 * no identity, no smoothing or expression regularisation (the video fit's initializer,
 * video_fitter.cu:30). Unknowns z = (epsilon[K], tau[3], u[3], s): the barrier method minimises
 * tau_lb s - sum log(G) - sum log(bound gaps) with G = s - (constraint gap) and stops once
 * s < -0.01 (every landmark inside its box by a margin). Sums over landmarks and constraint rows
 * (cuBLAS in the reference) are FP64 in a fixed order: rows in the order G_x-, G_y-, G_x+, G_y+,
 * landmarks ascending within each; the Hessian is an FMA chain over those rows. */

#define LM_ROWS (4 * O_NL)
#define LM_PI 3.14159265358979323846   /* M_PI of <math.h> (not declared under -std=c11) */

typedef struct {
    real G[LM_ROWS];          /* G_x-, G_y-, G_x+, G_y+ */
    real invG[LM_ROWS];       /* 1 / (1e-6 + G) */
    real nlog[LM_ROWS];       /* -log G */
    real *F;                  /* [LM_ROWS][n]: constraint rows of the barrier derivative */
    real *nWx, *nWy;          /* [O_NL][n - 1]: projection derivatives */
    real R[9], dR[27];
} lm_terms_t;

/* compute_nonrigid_shape + compute_Gs + the derivative kernels at z. */
static void lm_terms(const o_model *m, const o_frame *f, const real *z, int deriv, lm_terms_t *o)
{
    const int K = m->K, V = m->V, n = K + 7;
    const real *tau = z + K, s = z[K + 6];
    const real phix = f->phix, phiy = f->phiy, cx = f->cx, cy = f->cy, fs = f->face_size;
    o_rotation(z + K + 3, o->R, deriv ? o->dR : NULL);
    const real *R = o->R;
    real p[O_NL * 3], Rp[O_NL * 3];
    for (int i = 0; i < O_NL; ++i) {
        const int v = m->lis[i];
        for (int c = 0; c < 3; ++c) {
            const float *e = m->E + ((size_t)v * 3 + c) * K;
            real acc = 0;
            for (int k = 0; k < K; ++k) acc = RFMA((real)e[k], z[k], acc);
            p[i * 3 + c] = (real)m->mean[c * V + v] + acc;
        }
        for (int r = 0; r < 3; ++r)
            Rp[i * 3 + r] = (R[r] * p[i * 3] + R[r + 3] * p[i * 3 + 1]) + R[r + 6] * p[i * 3 + 2];
    }
    for (int i = 0; i < O_NL; ++i) {
        const real r1p = Rp[i * 3], r2p = Rp[i * 3 + 1], r3p = Rp[i * 3 + 2];
        const real xproj = phix * ((r1p + tau[0]) / (r3p + tau[2])) + cx;
        const real yproj = phiy * ((r2p + tau[1]) / (r3p + tau[2])) + cy;
        const real xl = f->xl[i], yl = f->yl[i];
        o->G[0 * O_NL + i] = s - ((xl + (real)f->bounds[0 * O_NL + i] * fs) - xproj);
        o->G[1 * O_NL + i] = s - ((yl + (real)f->bounds[1 * O_NL + i] * fs) - yproj);
        o->G[2 * O_NL + i] = s - ((xproj - (real)f->bounds[2 * O_NL + i] * fs) - xl);
        o->G[3 * O_NL + i] = s - ((yproj - (real)f->bounds[3 * O_NL + i] * fs) - yl);
    }
    for (int r = 0; r < LM_ROWS; ++r) {
        o->invG[r] = (real)1 / ((real)0.000001f + o->G[r]);
        o->nlog[r] = -RLOG(o->G[r]);
    }
    if (!deriv) return;
    for (int i = 0; i < O_NL; ++i) {
        const real px = p[i * 3], py = p[i * 3 + 1], pz = p[i * 3 + 2];
        const real vx = Rp[i * 3] + tau[0], vy = Rp[i * 3 + 1] + tau[1], vz = Rp[i * 3 + 2] + tau[2];
        const real ivz = (real)1 / vz, ivz2 = ivz * ivz;
        real *wx = o->nWx + (size_t)i * (n - 1), *wy = o->nWy + (size_t)i * (n - 1);
        const float *ex = m->E + (size_t)m->lis[i] * 3 * K;
        for (int k = 0; k < K; ++k) {
            real RIX = ex[k], RIY = ex[K + k], RIZ = ex[2 * K + k];
            real dvx = (RIX * R[0] + RIY * R[3]) + RIZ * R[6];
            real dvy = (RIX * R[1] + RIY * R[4]) + RIZ * R[7];
            real dvz = (RIX * R[2] + RIY * R[5]) + RIZ * R[8];
            wx[k] = (phix * ivz2) * (dvx * vz - dvz * vx);
            wy[k] = (phiy * ivz2) * (dvy * vz - dvz * vy);
        }
        wx[K + 0] = phix * ivz; wx[K + 1] = 0; wx[K + 2] = ((-phix) * vx) * ivz2;
        wy[K + 0] = 0; wy[K + 1] = phiy * ivz; wy[K + 2] = ((-phiy) * vy) * ivz2;
        for (int a = 0; a < 3; ++a) {
            const real *d = o->dR + 9 * a;
            real dvx = (d[0] * px + d[3] * py) + d[6] * pz;
            real dvy = (d[1] * px + d[4] * py) + d[7] * pz;
            real dvz = (d[2] * px + d[5] * py) + d[8] * pz;
            wx[K + 3 + a] = (phix * ivz2) * (vz * dvx - vx * dvz);
            wy[K + 3 + a] = (phiy * ivz2) * (vz * dvy - vy * dvz);
        }
        for (int a = 0; a < n - 1; ++a) {
            o->F[(size_t)(0 * O_NL + i) * n + a] = (-wx[a]) / o->G[0 * O_NL + i];
            o->F[(size_t)(1 * O_NL + i) * n + a] = (-wy[a]) / o->G[1 * O_NL + i];
            o->F[(size_t)(2 * O_NL + i) * n + a] = wx[a] / o->G[2 * O_NL + i];
            o->F[(size_t)(3 * O_NL + i) * n + a] = wy[a] / o->G[3 * O_NL + i];
        }
        for (int q = 0; q < 4; ++q) o->F[(size_t)(q * O_NL + i) * n + n - 1] = 0;
    }
}

/* tau_lb s + expression-bound and constraint barrier terms (evaluate_objective_function),
 * FP64 sums in the order of the reference's accumulations, rounded to REAL. */
static real lm_objective(const o_model *m, const real *z, real tau, const lm_terms_t *o)
{
    const int K = m->K;
    double acc = (double)(tau * z[K + 6]);
    double sl = 0.0, su = 0.0, sg = 0.0;
    for (int k = 0; k < K; ++k) sl += (double)(-RLOG(-((real)m->eps_lb[k] - z[k])));
    for (int k = 0; k < K; ++k) su += (double)(-RLOG(-(z[k] - (real)m->eps_ub[k])));
    for (int r = 0; r < LM_ROWS; ++r) sg += (double)o->nlog[r];
    acc += sl;
    acc += su;
    acc += sg;
    return (real)acc;
}

/* Gradient g [n] and Hessian H [n][n] (row-major, symmetric) of the barrier problem at the
 * terms o (compute_gradient_and_hessian with use_slack). */
static void lm_grad_hess(const o_model *m, const real *z, real tau, const lm_terms_t *o, real *g, real *H)
{
    const int K = m->K, n = K + 7, nb = n - 1;
    for (int a = 0; a < nb; ++a) {
        /* nablaF: the four rows of each landmark added elementwise (cublasSgeam), then summed
         * over the landmarks */
        double acc = 0.0;
        for (int i = 0; i < O_NL; ++i) {
            real e = o->F[(size_t)(0 * O_NL + i) * n + a];
            e = e + o->F[(size_t)(1 * O_NL + i) * n + a];
            e = e + o->F[(size_t)(2 * O_NL + i) * n + a];
            e = e + o->F[(size_t)(3 * O_NL + i) * n + a];
            acc += (double)e;
        }
        g[a] = (real)acc;
    }
    for (int k = 0; k < K; ++k) {              /* update_gradient (:915-929) */
        const real fub = z[k] - (real)m->eps_ub[k], flb = (real)m->eps_lb[k] - z[k];
        g[k] = g[k] + ((real)-1 / fub + (real)1 / flb);
    }
    {
        double acc = 0.0;
        for (int r = 0; r < LM_ROWS; ++r) acc += (double)o->invG[r];
        g[nb] = (real)(-acc);
        g[nb] = tau + g[nb];
    }
    for (int a = 0; a < nb; ++a)
        for (int b = 0; b <= a; ++b) {
            double acc = 0.0;
            for (int r = 0; r < LM_ROWS; ++r)
                acc = fma((double)o->F[(size_t)r * n + a], (double)o->F[(size_t)r * n + b], acc);
            H[(size_t)a * n + b] = H[(size_t)b * n + a] = (real)acc;
        }
    for (int k = 0; k < K; ++k) {              /* update_diagonal_of_hessian_wbounds (:932-949) */
        const real fub = z[k] - (real)m->eps_ub[k], flb = (real)m->eps_lb[k] - z[k];
        const real nu = (real)(-1.0 / ((double)fub + 1e-12));
        const real nl = (real)(1.0 / ((double)flb + 1e-12));
        H[(size_t)k * n + k] = H[(size_t)k * n + k] + (nu * nu + nl * nl);
    }
    for (int a = 0; a < nb; ++a) {             /* fill_for_nabla2F_dsdc + bottom and right */
        double acc = 0.0;
        for (int i = 0; i < O_NL; ++i) {
            const real gxm = o->G[i], gym = o->G[O_NL + i], gxp = o->G[2 * O_NL + i], gyp = o->G[3 * O_NL + i];
            const real wx = o->nWx[(size_t)i * nb + a], wy = o->nWy[(size_t)i * nb + a];
            real e = (-wx) / (gxp * gxp) - wy / (gyp * gyp);
            e = e + wx / (gxm * gxm);
            e = e + wy / (gym * gym);
            acc += (double)e;
        }
        H[(size_t)nb * n + a] = H[(size_t)a * n + nb] = (real)acc;
    }
    {
        double acc = 0.0;
        for (int r = 0; r < LM_ROWS; ++r) acc = fma((double)o->invG[r], (double)o->invG[r], acc);
        H[(size_t)nb * n + nb] = (real)acc;
    }
}

/* Euler angles in degrees of the rotation (RotationComputer::compute_euler_angles,
 * rotation_header.cu:421-449, with RAD2DEG of constants.h:59): atan2 in double, rounded. */
static void lm_euler_deg(const float *R, float *yaw, float *pitch, float *roll)
{
    const float c = sqrtf(R[5] * R[5] + R[8] * R[8]);
    float y, p, r;
    if (!(c < 1e-6f)) {
        r = (float)atan2((double)R[1], (double)R[0]);
        y = (float)atan2((double)-R[2], (double)c);
        p = (float)atan2((double)R[5], (double)R[8]);
    } else {
        r = (float)atan2((double)-R[7], (double)R[4]);
        y = (float)atan2((double)-R[2], (double)c);
        p = 0.0f;
    }
    *yaw = (float)((double)(y * 180.0f) / LM_PI);
    *pitch = (float)((double)(p * 180.0f) / LM_PI);
    *roll = (float)((double)(r * 180.0f) / LM_PI);
}

/* The start rotation of the second orthographic fit when the first one converged to a mirrored
 * solution (sigma_x < 0, logbarrier_initializer.cu:1872-1896): the Euler angles (roll, -pitch,
 * -yaw) as a rotation R = Rz Ry Rx (eulerAnglesToRotationMatrix, newfuncs.cu:720-747) turned
 * into an axis-angle vector (cv::Rodrigues). OpenCV's float matrix product and its Rodrigues
 * (an SVD re-orthonormalisation, then the axis from the skew part) are evaluated here in
 * double from the same float angles: theta = acos((trace - 1) / 2), axis = (R32 - R23,
 * R13 - R31, R21 - R12) / (2 sin theta), and for theta near pi the axis from the diagonal. */
static void lm_flip_rotation(float yaw, float pitch, float roll, float *u)
{
    const float th[3] = {(float)(((double)roll * LM_PI) / 180.0), (float)(((double)(-pitch) * LM_PI) / 180.0),
                         (float)(((double)(-yaw) * LM_PI) / 180.0)};
    /* cos and sin of the float angles in double, rounded to float (the float overloads the
     * reference calls) */
    const double c0 = (float)cos((double)th[0]), s0 = (float)sin((double)th[0]);
    const double c1 = (float)cos((double)th[1]), s1 = (float)sin((double)th[1]);
    const double c2 = (float)cos((double)th[2]), s2 = (float)sin((double)th[2]);
    const double Rx[9] = {1, 0, 0, 0, c0, -s0, 0, s0, c0};       /* row-major */
    const double Ry[9] = {c1, 0, s1, 0, 1, 0, -s1, 0, c1};
    const double Rz[9] = {c2, -s2, 0, s2, c2, 0, 0, 0, 1};
    double T[9], R[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T[i * 3 + j] = 0;
            for (int k = 0; k < 3; ++k) T[i * 3 + j] += Ry[i * 3 + k] * Rx[k * 3 + j];
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            R[i * 3 + j] = 0;
            for (int k = 0; k < 3; ++k) R[i * 3 + j] += Rz[i * 3 + k] * T[k * 3 + j];
        }
    const double rx = R[7] - R[5], ry = R[2] - R[6], rz = R[3] - R[1];
    const double sn = 0.5 * sqrt(rx * rx + ry * ry + rz * rz);
    double cs = 0.5 * (R[0] + R[4] + R[8] - 1.0);
    cs = cs > 1.0 ? 1.0 : (cs < -1.0 ? -1.0 : cs);
    const double theta = acos(cs);
    double out[3];
    if (sn < 1e-5) {
        if (cs > 0) { out[0] = out[1] = out[2] = 0.0; }
        else {
            double ax = sqrt((R[0] + 1) * 0.5), ay = sqrt((R[4] + 1) * 0.5), az = sqrt((R[8] + 1) * 0.5);
            if (R[1] < 0) ay = -ay;
            if (R[2] < 0) az = -az;
            if (fabs(ax) < fabs(ay) && fabs(ax) < fabs(az) && (R[5] > 0) != (ay * az > 0)) az = -az;
            out[0] = ax * theta; out[1] = ay * theta; out[2] = az * theta;
        }
    } else {
        const double v = theta / (2.0 * sn);
        out[0] = rx * v; out[1] = ry * v; out[2] = rz * v;
    }
    for (int k = 0; k < 3; ++k) u[k] = (float)out[k];
}

/* Landmark initialisation of one frame. p0L [3][51]: the orthographic step's landmark points
 * (p0L_mat.dat). Writes z_out [K+6] (epsilon, tau, u) and the final slack; returns 1 when
 * the barrier method reached s < -0.01 (fit_success), 0 otherwise. *newton counts the
 * Newton iterations, *orth_flip whether the mirrored-solution branch ran. */
int o_landmark_init_f(const o_model *m, const o_frame *f, const float *p0L, float *z_out, float *slack_out,
                      int *newton, int *orth_flip)
{
    const int K = m->K, n = K + 7;
    /* initialize_with_orthographic_t (:1862-1918) */
    float xo[ORTH_N], Rl[9], yaw, pitch, roll;
    o_orthographic_f(f->xl, f->yl, p0L, xo, Rl);
    lm_euler_deg(Rl, &yaw, &pitch, &roll);
    *orth_flip = 0;
    if (xo[2] < 0) {
        float u0[3];
        lm_flip_rotation(yaw, pitch, roll, u0);
        xo[0] = -xo[0];
        xo[2] = -xo[2];
        xo[4] = u0[0]; xo[5] = u0[1]; xo[6] = u0[2];
        orth_fit(f->xl, f->yl, p0L, xo, Rl);
        *orth_flip = 1;
    }
    float xm = 0.0f, ym = 0.0f;                 /* thrust::reduce on the host, then / 51 */
    for (int i = 0; i < O_NL; ++i) { xm += f->xl[i]; ym += f->yl[i]; }
    xm = xm / (float)O_NL;
    ym = ym / (float)O_NL;
    /* initialize_kernel (:31-51) */
    const float tz = (float)((double)f->phix / ((double)(fabsf(xo[2]) + fabsf(xo[3])) * 0.5));
    real *z = (real *)calloc((size_t)n, sizeof(real)), *zt = (real *)calloc((size_t)n, sizeof(real));
    z[K + 2] = tz;
    z[K + 0] = (float)((tz * (xm - f->cx)) / f->phix);
    z[K + 1] = (float)((tz * (ym - f->cy)) / f->phiy);
    z[K + 3] = xo[4]; z[K + 4] = xo[5]; z[K + 5] = xo[6];
    lm_terms_t o;
    o.F = (real *)malloc(sizeof(real) * LM_ROWS * (size_t)n);
    o.nWx = (real *)malloc(sizeof(real) * O_NL * (size_t)n);
    o.nWy = (real *)malloc(sizeof(real) * O_NL * (size_t)n);
    real *H = (real *)malloc(sizeof(real) * (size_t)n * n), *g = (real *)malloc(sizeof(real) * n);
    real *d = (real *)malloc(sizeof(real) * n);
    /* set_minimal_slack (:1041-1092): with s = 0, s0 = 5 - min G */
    z[K + 6] = 0;
    lm_terms(m, f, z, 0, &o);
    real gmin = o.G[0];
    for (int r = 1; r < LM_ROWS; ++r) gmin = o.G[r] < gmin ? o.G[r] : gmin;
    z[K + 6] = (real)5.0f - gmin;
    /* fit_model (:1095-1269) */
    real tau = (real)10.0f;
    int success = 0, iters = 0;
    for (int stage = 0; stage < 5 && !success; ++stage) {
        tau = tau * (real)10.0f;
        int terminate = 0;
        for (int it = 0; it < 100 && !terminate; ++it) {
            if (z[K + 6] < (real)-0.01f) { success = 1; break; }
            lm_terms(m, f, z, 1, &o);
            const real obj = lm_objective(m, z, tau, &o);
            lm_grad_hess(m, z, tau, &o, g, H);
            ++iters;
            if (!solve(H, g, n, d, 0.0f)) { terminate = 1; break; }
            real t = (real)1.0f;
            for (int inner = 0; inner < 100; ++inner) {
                if (t < (real)0.01f) { terminate = 1; break; }
                for (int a = 0; a < n; ++a) zt[a] = z[a] + t * d[a];
                lm_terms(m, f, zt, 0, &o);
                const real ot = lm_objective(m, zt, tau, &o);
                if (ot < obj) { memcpy(z, zt, sizeof(real) * n); break; }
                t = t * (real)0.5f;
            }
        }
    }
    for (int a = 0; a < K + 6; ++a) z_out[a] = (float)z[a];
    *slack_out = (float)z[K + 6];
    *newton = iters;
    free(o.F); free(o.nWx); free(o.nWy); free(H); free(g); free(d); free(z); free(zt);
    return success;
}

/* ------------------------------------------------------------------------------------ */
/* Renderer::compute_nonrigid_shape_identityonly and compute_texture (renderer.cu:866-883,
 * 941-951): mean[c][v] = mean0[c][v] + (sequential fmaf chain over k of id[c][v][k] alpha[k])
 * and tex[v] = tex0[v] + (the same over TEX[v][k] beta[k]); n_id or n_tex 0 leaves a copy. The
 * reference's cublasSgemv order is the library's; this order is the contract shared with the
 * device. FP32 in both builds. */
void o_apply_identity(int V, int KA, int KB, const float *mean0, const float *I, const float *alpha,
                      const float *tex0, const float *T, const float *beta, float *mean, float *tex)
{
    for (int r = 0; r < 3 * V; ++r) {
        float acc = 0.0f;
        for (int k = 0; k < KA; ++k) acc = fmaf(I[(size_t)r * KA + k], alpha[k], acc);
        mean[r] = KA ? mean0[r] + acc : mean0[r];
    }
    for (int v = 0; v < V; ++v) {
        float acc = 0.0f;
        for (int k = 0; k < KB; ++k) acc = fmaf(T[(size_t)v * KB + k], beta[k], acc);
        tex[v] = KB ? tex0[v] + acc : tex0[v];
    }
}
