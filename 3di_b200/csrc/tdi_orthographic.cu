// Orthographic pose initialisation of many frames (OrthographicInitializer::fit_model,
// orthographic_initializer.cu:243-380), a warp per frame.
//
// Per frame: x = (tau_x, tau_y, sigma_x, sigma_y, u1, u2, u3) from (0, 0, 15, 15, 0, 0, 0.05)
// (:152-167); residuals sigma_x (R p_i + tau)_x - xbar_i and sigma_y (R p_i + tau)_y - ybar_i
// of the model's 51 landmark points p (p0L) against the centred landmarks; Gauss-Newton with
// the 7 x 7 system solved in FP64; Armijo line search (alpha 0.4, beta 0.5) until t < 0.1,
// which ends the fit; at most 100 outer iterations. FP32 as the reference, its library
// calls in a fixed order shared with the oracle: landmark means as sequential float sums,
// R p as ((R0 p0 + R3 p1) + R6 p2), J^T J, J^T e and the dot products as float fused
// multiply-add chains over the 102 residual rows in order (x rows, then y rows), the
// Cholesky factor by left-looking dot products in increasing k, forward substitution in
// increasing k, back substitution in decreasing k.

namespace tdi {

constexpr int OR_WARPS = 4;                 // frames per block
constexpr int OR_N = 7;
constexpr int OR_ROWS = 2 * NL;

struct OrthWarp {
    float xb[NL], yb[NL];                   // centred landmarks
    float W[OR_N][OR_ROWS];                 // Jacobian columns
    float e[OR_ROWS];                       // residuals (of the point, then of each trial)
    float R[9], dR[27], Rt[9], dRt[27];     // rotation of the point and of the last trial
    float x[OR_N], xs[OR_N], sd[OR_N], dg[OR_N], JTJ[OR_N * OR_N];
    float obj;
    int accept;
};

__device__ __forceinline__ void orth_rp(const float *R, const float *p0L, int i, float *r)
{
    const float p0 = p0L[i], p1 = p0L[NL + i], p2 = p0L[2 * NL + i];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] = (R[k] * p0 + R[3 + k] * p1) + R[6 + k] * p2;
}

// d = -(H^-1 g) for the 7 x 7 system, FP64 (solver.h:70-105); NaN when H is not positive definite.
__device__ void orth_solve(const float *H, const float *g, float *d)
{
    double L[OR_N * OR_N], y[OR_N];
    for (int i = 0; i < OR_N * OR_N; ++i) L[i] = (double)H[i];
    bool ok = true;
    for (int j = 0; j < OR_N && ok; ++j) {
        double s = L[j * OR_N + j];
        for (int k = 0; k < j; ++k) s -= L[k * OR_N + j] * L[k * OR_N + j];
        if (!(s > 0.0)) { ok = false; break; }
        const double ljj = sqrt(s);
        L[j * OR_N + j] = ljj;
        for (int i = j + 1; i < OR_N; ++i) {
            double t = L[j * OR_N + i];
            for (int k = 0; k < j; ++k) t -= L[k * OR_N + i] * L[k * OR_N + j];
            L[j * OR_N + i] = t / ljj;
        }
    }
    if (!ok) {
        for (int i = 0; i < OR_N; ++i) d[i] = __int_as_float(0x7fc00000);
        return;
    }
    for (int i = 0; i < OR_N; ++i) {
        double t = (double)g[i];
        for (int k = 0; k < i; ++k) t -= L[k * OR_N + i] * y[k];
        y[i] = t / L[i * OR_N + i];
    }
    for (int i = OR_N - 1; i >= 0; --i) {
        double t = y[i];
        for (int k = OR_N - 1; k > i; --k) t -= L[i * OR_N + k] * y[k];
        y[i] = t / L[i * OR_N + i];
    }
    for (int i = 0; i < OR_N; ++i) d[i] = (float)(-y[i]);
}

// x_start: NULL for the reference's start point (reset_orthographic), else [F][7] start points
// (fit_model with reset_variables = false); run: NULL, or [F] flags selecting the frames fitted.
__global__ void __launch_bounds__(OR_WARPS * 32) k_orthographic(const float *xl, const float *yl, const float *p0L,
                                                                int F, float *x_out, float *R_out, int32_t *iters,
                                                                const float *x_start, const int32_t *run)
{
    __shared__ OrthWarp sw[OR_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int f = blockIdx.x * OR_WARPS + warp;
    if (f >= F) return;
    if (run && !run[f]) return;
    OrthWarp &w = sw[warp];
    const float *xf = xl + (size_t)f * NL, *yf = yl + (size_t)f * NL;
    float xm = 0.0f, ym = 0.0f;
    if (lane == 0) {
        for (int i = 0; i < NL; ++i) { xm += xf[i]; ym += yf[i]; }
        xm = xm / (float)NL;
        ym = ym / (float)NL;
        const float x0[OR_N] = {0.0f, 0.0f, 15.0f, 15.0f, 0.0f, 0.0f, 0.05f};
        for (int n = 0; n < OR_N; ++n) w.x[n] = x_start ? x_start[(size_t)f * OR_N + n] : x0[n];
        for (int k = 0; k < 9; ++k) w.Rt[k] = 0.0f;
    }
    xm = __shfl_sync(0xffffffffu, xm, 0);
    ym = __shfl_sync(0xffffffffu, ym, 0);
    for (int i = lane; i < NL; i += 32) { w.xb[i] = xf[i] - xm; w.yb[i] = yf[i] - ym; }
    __syncwarp();
    bool terminate = false;
    int q;
    for (q = 0; q < 100; ++q) {
        if (terminate) break;
        if (lane == 0) rotation(w.x + 4, w.R, w.dR);
        __syncwarp();
        for (int i = lane; i < NL; i += 32) {
            float rp[3], d[3][3];
            orth_rp(w.R, p0L, i, rp);
#pragma unroll
            for (int a = 0; a < 3; ++a) orth_rp(w.dR + 9 * a, p0L, i, d[a]);
            const float tx = w.x[0], ty = w.x[1], sx = w.x[2], sy = w.x[3];
            w.W[0][i] = sx;         w.W[0][NL + i] = 0.0f;
            w.W[1][i] = 0.0f;       w.W[1][NL + i] = sy;
            w.W[2][i] = tx + rp[0]; w.W[2][NL + i] = 0.0f;
            w.W[3][i] = 0.0f;       w.W[3][NL + i] = ty + rp[1];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                w.W[4 + a][i] = sx * d[a][0];
                w.W[4 + a][NL + i] = sy * d[a][1];
            }
            w.e[i] = sx * (rp[0] + tx) - w.xb[i];
            w.e[NL + i] = sy * (rp[1] + ty) - w.yb[i];
        }
        __syncwarp();
        for (int k = lane; k < OR_N * OR_N; k += 32) {
            const int a = k % OR_N, b = k / OR_N;
            float s = 0.0f;
            for (int r = 0; r < OR_ROWS; ++r) s = fmaf(w.W[a][r], w.W[b][r], s);
            w.JTJ[k] = s;
        }
        if (lane < OR_N) {
            float s = 0.0f;
            for (int r = 0; r < OR_ROWS; ++r) s = fmaf(w.W[lane][r], w.e[r], s);
            w.dg[lane] = s;
        } else if (lane == OR_N) {
            float s = 0.0f;
            for (int r = 0; r < OR_ROWS; ++r) s = fmaf(w.e[r], w.e[r], s);
            w.obj = s;
        }
        __syncwarp();
        if (lane == 0) orth_solve(w.JTJ, w.dg, w.sd);
        __syncwarp();
        float t = 1.0f;
        for (int inner = 0; inner < 1000; ++inner) {
            if (t < 0.1f) { terminate = true; break; }
            if (lane == 0) {
                for (int n = 0; n < OR_N; ++n) w.xs[n] = w.x[n] + t * w.sd[n];
                rotation(w.xs + 4, w.Rt, w.dRt);
            }
            __syncwarp();
            for (int i = lane; i < NL; i += 32) {
                float rp[3];
                orth_rp(w.Rt, p0L, i, rp);
                w.e[i] = w.xs[2] * (rp[0] + w.xs[0]) - w.xb[i];
                w.e[NL + i] = w.xs[3] * (rp[1] + w.xs[1]) - w.yb[i];
            }
            __syncwarp();
            if (lane == 0) {
                float objt = 0.0f, tmp = 0.0f;
                for (int r = 0; r < OR_ROWS; ++r) objt = fmaf(w.e[r], w.e[r], objt);
                for (int n = 0; n < OR_N; ++n) tmp = fmaf(w.sd[n], w.dg[n], tmp);
                tmp *= 0.4f * t;
                w.accept = objt < w.obj + tmp;
                if (w.accept)
                    for (int n = 0; n < OR_N; ++n) w.x[n] = w.xs[n];
            }
            __syncwarp();
            if (w.accept) break;
            t = t * 0.5f;
        }
    }
    if (lane == 0) {
        for (int n = 0; n < OR_N; ++n) x_out[(size_t)f * OR_N + n] = w.x[n];
        for (int k = 0; k < 9; ++k) R_out[(size_t)f * 9 + k] = w.Rt[k];
        iters[f] = q;
    }
}

}  // namespace tdi
