// Landmark initialisation of many frames: the step VideoFitter::fit_to_video_frame runs before
// the image fit (video_fitter.cu:456-500). Per frame:
//   1. the orthographic pose fit to the landmarks (k_orthographic, a warp per frame); when it
//      ends on a mirrored solution (sigma_x < 0) the start is rebuilt from the Euler angles of
//      its rotation and the fit runs again from there (initialize_with_orthographic_t,
//      logbarrier_initializer.cu:1862-1896; k_lm_flip);
//   2. the perspective start: tau_z from the orthographic scales, tau_x, tau_y from the
//      landmark centre, the orthographic rotation, zero expressions (initialize_kernel, :31-51);
//   3. the smallest slack that makes every landmark constraint hold by 5 (set_minimal_slack,
//      :1041-1092);
//   4. the barrier method with a slack variable (fit_model, :1095-1269): five stages with the
//      barrier weight multiplied by 10 (100 ... 1e6), up to 100 Newton steps each on
//      z = (epsilon, tau, u, s) with an FP64 Cholesky solve and a backtracking line search
//      (halving from t = 1 while the objective does not decrease, stopping below t = 0.01),
//      until s < -0.01: every landmark inside its box with a margin.
// Steps 2-4 run as one block per frame with every iteration on the device. Arithmetic as the
// oracle (o_landmark_init_f): FP32 elementwise in the reference's operand order, sums over
// landmarks and constraint rows in FP64 in a fixed order (rows G_x-, G_y-, G_x+, G_y+,
// landmarks ascending), the Hessian as an FP64 fused multiply-add chain over those rows, the
// Cholesky factor left-looking with dot products in increasing k.

namespace tdi {

constexpr int LM_THREADS = 256;
constexpr int LM_ROWS = 4 * NL;

// Euler angles in degrees of a rotation (rotation_header.cu:421-449, RAD2DEG).
__device__ void lm_euler_deg(const float *R, float *yaw, float *pitch, float *roll)
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
    *yaw = (float)((double)(y * 180.0f) / 3.14159265358979323846);
    *pitch = (float)((double)(p * 180.0f) / 3.14159265358979323846);
    *roll = (float)((double)(r * 180.0f) / 3.14159265358979323846);
}

// New orthographic start for frames whose fit ended with sigma_x < 0: rotation from the angles
// (roll, -pitch, -yaw) (eulerAnglesToRotationMatrix, newfuncs.cu:720-747) turned into an
// axis-angle vector (cv::Rodrigues), both evaluated in double from the float angles; tau_x and
// sigma_x change sign. run[f] selects the frames to fit again.
__global__ void k_lm_flip(int F, float *xo, const float *Ro, int32_t *run)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    float *x = xo + (size_t)f * 7;
    run[f] = 0;
    if (!(x[2] < 0.0f)) return;
    float yaw, pitch, roll;
    lm_euler_deg(Ro + (size_t)f * 9, &yaw, &pitch, &roll);
    const double PI = 3.14159265358979323846;
    const float th[3] = {(float)(((double)roll * PI) / 180.0), (float)(((double)(-pitch) * PI) / 180.0),
                         (float)(((double)(-yaw) * PI) / 180.0)};
    const double c0 = (float)cos((double)th[0]), s0 = (float)sin((double)th[0]);
    const double c1 = (float)cos((double)th[1]), s1 = (float)sin((double)th[1]);
    const double c2 = (float)cos((double)th[2]), s2 = (float)sin((double)th[2]);
    const double Rx[9] = {1, 0, 0, 0, c0, -s0, 0, s0, c0};
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
        if (cs > 0) {
            out[0] = out[1] = out[2] = 0.0;
        } else {
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
    x[0] = -x[0];
    x[2] = -x[2];
    x[4] = (float)out[0]; x[5] = (float)out[1]; x[6] = (float)out[2];
    run[f] = 1;
}

struct LmShared {
    float G[LM_ROWS], invG[LM_ROWS], nlog[LM_ROWS];
    float p[NL * 3], Rp[NL * 3];
    float R[9], dR[27];
    float obj, ot, tau, t;
    int flag;            // solve failure
};

constexpr size_t LM_HDR = (sizeof(LmShared) + 15) / 16 * 16;   // keeps the FP64 factor 16-byte aligned
constexpr int LM_MAXN = 136;                                      // unknowns (K + 7) at most

__host__ __device__ __forceinline__ size_t lm_smem(int K)
{
    const int n = K + 7;
    // z, zt, d, g [n]; H [n][n]; F [LM_ROWS][n] (reused as the FP64 factor [n][n]); nW [2][NL][n-1]
    const size_t fl = (size_t)4 * n + (size_t)n * n + (size_t)2 * NL * (n - 1);
    const size_t fbytes = (size_t)LM_ROWS * n * sizeof(float);
    const size_t lbytes = (size_t)n * n * sizeof(double);
    return LM_HDR + ((fbytes > lbytes ? fbytes : lbytes) + 15) / 16 * 16 + fl * sizeof(float);
}

// Constraint terms at z (compute_nonrigid_shape + compute_Gs, :456-520, 2124-2140) and, with
// deriv, the derivative rows (fill_optimization_dc_landmark, :587-697,
// fill_optimization_dI_depsilon_landmark, :836-912).
__device__ void lm_terms(const DModel &m, const float *xl, const float *yl, const float *bd, float fs,
                         const float *cam, const float *z, bool deriv, LmShared &s, float *F, float *nWx,
                         float *nWy)
{
    const int K = m.K, KP = m.KP, V = m.V, n = K + 7, nb = n - 1, tid = threadIdx.x;
    if (tid == 0) rotation(z + K + 3, s.R, s.dR);
    __syncthreads();
    if (tid < NL * 3) {
        const int i = tid / 3, c = tid - 3 * i, v = m.lis[i];
        const float *e = m.E + ((size_t)v * 3 + c) * KP;
        float acc = 0.0f;
        for (int k = 0; k < K; ++k) acc = fmaf(e[k], z[k], acc);
        s.p[tid] = m.mean[(size_t)c * V + v] + acc;
    }
    __syncthreads();
    const float *R = s.R;
    const float sl = z[nb];
    if (tid < NL) {
        const int i = tid;
        const float *p = s.p + 3 * i;
        for (int r = 0; r < 3; ++r) s.Rp[3 * i + r] = (R[r] * p[0] + R[r + 3] * p[1]) + R[r + 6] * p[2];
        const float r1p = s.Rp[3 * i], r2p = s.Rp[3 * i + 1], r3p = s.Rp[3 * i + 2];
        const float xproj = cam[0] * ((r1p + z[K]) / (r3p + z[K + 2])) + cam[2];
        const float yproj = cam[1] * ((r2p + z[K + 1]) / (r3p + z[K + 2])) + cam[3];
        s.G[0 * NL + i] = sl - ((xl[i] + bd[0 * NL + i] * fs) - xproj);
        s.G[1 * NL + i] = sl - ((yl[i] + bd[1 * NL + i] * fs) - yproj);
        s.G[2 * NL + i] = sl - ((xproj - bd[2 * NL + i] * fs) - xl[i]);
        s.G[3 * NL + i] = sl - ((yproj - bd[3 * NL + i] * fs) - yl[i]);
        for (int q = 0; q < 4; ++q) {
            const float G = s.G[q * NL + i];
            s.invG[q * NL + i] = 1.0f / (0.000001f + G);
            s.nlog[q * NL + i] = -(float)log((double)G);
        }
    }
    __syncthreads();
    if (!deriv) return;
    const float phix = cam[0], phiy = cam[1];
    // projection derivatives: expression columns, then the six pose columns
    for (int w = tid; w < NL * (K + 6); w += LM_THREADS) {
        const int i = w / (K + 6), a = w - i * (K + 6);
        const float vx = s.Rp[3 * i] + z[K], vy = s.Rp[3 * i + 1] + z[K + 1], vz = s.Rp[3 * i + 2] + z[K + 2];
        const float ivz = 1.0f / vz, ivz2 = ivz * ivz;
        float wx, wy;
        if (a < K) {
            const float *ex = m.E + (size_t)m.lis[i] * 3 * KP;
            const float RIX = ex[a], RIY = ex[KP + a], RIZ = ex[2 * KP + a];
            const float dvx = (RIX * R[0] + RIY * R[3]) + RIZ * R[6];
            const float dvy = (RIX * R[1] + RIY * R[4]) + RIZ * R[7];
            const float dvz = (RIX * R[2] + RIY * R[5]) + RIZ * R[8];
            wx = (phix * ivz2) * (dvx * vz - dvz * vx);
            wy = (phiy * ivz2) * (dvy * vz - dvz * vy);
        } else if (a == K) {
            wx = phix * ivz; wy = 0.0f;
        } else if (a == K + 1) {
            wx = 0.0f; wy = phiy * ivz;
        } else if (a == K + 2) {
            wx = ((-phix) * vx) * ivz2; wy = ((-phiy) * vy) * ivz2;
        } else {
            const float *d = s.dR + 9 * (a - K - 3);
            const float px = s.p[3 * i], py = s.p[3 * i + 1], pz = s.p[3 * i + 2];
            const float dvx = (d[0] * px + d[3] * py) + d[6] * pz;
            const float dvy = (d[1] * px + d[4] * py) + d[7] * pz;
            const float dvz = (d[2] * px + d[5] * py) + d[8] * pz;
            wx = (phix * ivz2) * (vz * dvx - vx * dvz);
            wy = (phiy * ivz2) * (vz * dvy - vy * dvz);
        }
        nWx[(size_t)i * nb + a] = wx;
        nWy[(size_t)i * nb + a] = wy;
        F[(size_t)(0 * NL + i) * n + a] = (-wx) / s.G[0 * NL + i];
        F[(size_t)(1 * NL + i) * n + a] = (-wy) / s.G[1 * NL + i];
        F[(size_t)(2 * NL + i) * n + a] = wx / s.G[2 * NL + i];
        F[(size_t)(3 * NL + i) * n + a] = wy / s.G[3 * NL + i];
    }
    for (int r = tid; r < LM_ROWS; r += LM_THREADS) F[(size_t)r * n + nb] = 0.0f;
    __syncthreads();
}

// tau s + expression-bound and constraint barrier terms, FP64 sums, rounded (thread 0).
__device__ float lm_objective(const DModel &m, const float *z, float tau, const LmShared &s)
{
    const int K = m.K;
    const float *lb = m.eps_b, *ub = m.eps_b + K;
    double acc = (double)(tau * z[K + 6]);
    double sl = 0.0, su = 0.0, sg = 0.0;
    for (int k = 0; k < K; ++k) sl += (double)(-(float)log((double)(-(lb[k] - z[k]))));
    for (int k = 0; k < K; ++k) su += (double)(-(float)log((double)(-(z[k] - ub[k]))));
    for (int r = 0; r < LM_ROWS; ++r) sg += (double)s.nlog[r];
    acc += sl;
    acc += su;
    acc += sg;
    return (float)acc;
}

__global__ void __launch_bounds__(LM_THREADS) k_landmark_init(DModel m, DBatch b, const float *xo,
                                                              int32_t *success_out, float *slack_out,
                                                              int32_t *iters_out)
{
    extern __shared__ __align__(16) unsigned char lm_raw[];
    LmShared &s = *reinterpret_cast<LmShared *>(lm_raw);
    const int K = m.K, n = K + 7, nb = n - 1, tid = threadIdx.x;
    const size_t fbytes = (size_t)LM_ROWS * n * sizeof(float), lbytes = (size_t)n * n * sizeof(double);
    unsigned char *big = lm_raw + LM_HDR;
    float *F = reinterpret_cast<float *>(big);
    double *Lf = reinterpret_cast<double *>(big);            // the factor, after F is used
    float *z = reinterpret_cast<float *>(big + ((fbytes > lbytes ? fbytes : lbytes) + 15) / 16 * 16);
    float *zt = z + n, *d = zt + n, *g = d + n, *H = g + n;
    float *nWx = H + (size_t)n * n, *nWy = nWx + (size_t)NL * nb;
    const int f = blockIdx.x;
    const float *xl = b.xl + (size_t)f * NL, *yl = b.yl + (size_t)f * NL;
    const float *bd = b.bounds + (size_t)f * 4 * NL, *cam = b.cam + (size_t)f * 4;
    const float fs = b.face_size[f];
    const float *lb = m.eps_b, *ub = m.eps_b + K;
    // perspective start (initialize_kernel) and zero expressions
    for (int a = tid; a < n; a += LM_THREADS) z[a] = 0.0f;
    __syncthreads();
    if (tid == 0) {
        const float *x7 = xo + (size_t)f * 7;
        float xm = 0.0f, ym = 0.0f;
        for (int i = 0; i < NL; ++i) { xm += xl[i]; ym += yl[i]; }
        xm = xm / (float)NL;
        ym = ym / (float)NL;
        const float tz = (float)((double)cam[0] / ((double)(fabsf(x7[2]) + fabsf(x7[3])) * 0.5));
        z[K + 2] = tz;
        z[K + 0] = (tz * (xm - cam[2])) / cam[0];
        z[K + 1] = (tz * (ym - cam[3])) / cam[1];
        z[K + 3] = x7[4]; z[K + 4] = x7[5]; z[K + 5] = x7[6];
    }
    __syncthreads();
    // minimal slack: s0 = 5 - min G at s = 0
    lm_terms(m, xl, yl, bd, fs, cam, z, false, s, F, nWx, nWy);
    if (tid == 0) {
        float gmin = s.G[0];
        for (int r = 1; r < LM_ROWS; ++r) gmin = s.G[r] < gmin ? s.G[r] : gmin;
        z[nb] = 5.0f - gmin;
        s.tau = 10.0f;
    }
    __syncthreads();
    int success = 0, iters = 0;
    for (int stage = 0; stage < 5 && !success; ++stage) {
        if (tid == 0) s.tau = s.tau * 10.0f;
        __syncthreads();
        const float tau = s.tau;
        bool terminate = false;
        for (int it = 0; it < 100 && !terminate; ++it) {
            if (z[nb] < -0.01f) { success = 1; break; }
            lm_terms(m, xl, yl, bd, fs, cam, z, true, s, F, nWx, nWy);
            if (tid == 0) s.obj = lm_objective(m, z, tau, s);
            // gradient
            for (int a = tid; a < nb; a += LM_THREADS) {
                double acc = 0.0;
                for (int i = 0; i < NL; ++i) {
                    float e = F[(size_t)(0 * NL + i) * n + a];
                    e = e + F[(size_t)(1 * NL + i) * n + a];
                    e = e + F[(size_t)(2 * NL + i) * n + a];
                    e = e + F[(size_t)(3 * NL + i) * n + a];
                    acc += (double)e;
                }
                float ga = (float)acc;
                if (a < K) {
                    const float fub = z[a] - ub[a], flb = lb[a] - z[a];
                    ga = ga + (-1.0f / fub + 1.0f / flb);
                }
                g[a] = ga;
            }
            if (tid == LM_THREADS - 1) {
                double acc = 0.0;
                for (int r = 0; r < LM_ROWS; ++r) acc += (double)s.invG[r];
                const float gs = (float)(-acc);
                g[nb] = tau + gs;
            }
            // Hessian: the lower triangle of the constraint block, one entry per item
            const int ntri = nb * (nb + 1) / 2;
            for (int w = tid; w < ntri; w += LM_THREADS) {
                int a = (int)((sqrt(8.0 * w + 1.0) - 1.0) * 0.5);
                while ((a + 1) * (a + 2) / 2 <= w) ++a;
                while (a * (a + 1) / 2 > w) --a;
                const int bcol = w - a * (a + 1) / 2;
                double acc = 0.0;
                for (int r = 0; r < LM_ROWS; ++r)
                    acc = fma((double)F[(size_t)r * n + a], (double)F[(size_t)r * n + bcol], acc);
                float hv = (float)acc;
                if (a == bcol && a < K) {
                    const float fub = z[a] - ub[a], flb = lb[a] - z[a];
                    const float nu = (float)(-1.0 / ((double)fub + 1e-12));
                    const float nl = (float)(1.0 / ((double)flb + 1e-12));
                    hv = hv + (nu * nu + nl * nl);
                }
                H[(size_t)a * n + bcol] = hv;
                H[(size_t)bcol * n + a] = hv;
            }
            for (int a = tid; a < nb; a += LM_THREADS) {
                double acc = 0.0;
                for (int i = 0; i < NL; ++i) {
                    const float gxm = s.G[i], gym = s.G[NL + i], gxp = s.G[2 * NL + i], gyp = s.G[3 * NL + i];
                    const float wx = nWx[(size_t)i * nb + a], wy = nWy[(size_t)i * nb + a];
                    float e = (-wx) / (gxp * gxp) - wy / (gyp * gyp);
                    e = e + wx / (gxm * gxm);
                    e = e + wy / (gym * gym);
                    acc += (double)e;
                }
                H[(size_t)nb * n + a] = (float)acc;
                H[(size_t)a * n + nb] = (float)acc;
            }
            if (tid == LM_THREADS - 2) {
                double acc = 0.0;
                for (int r = 0; r < LM_ROWS; ++r) acc = fma((double)s.invG[r], (double)s.invG[r], acc);
                H[(size_t)nb * n + nb] = (float)acc;
            }
            __syncthreads();
            ++iters;
            // FP64 Cholesky (solver.h:70-105), left-looking; the factor overwrites F
            for (int i = tid; i < n * n; i += LM_THREADS) Lf[i] = (double)H[i];
            if (tid == 0) s.flag = 0;
            __syncthreads();
            for (int j = 0; j < n; ++j) {
                if (tid == 0) {
                    double sj = Lf[(size_t)j * n + j];
                    for (int k = 0; k < j; ++k) sj -= Lf[(size_t)k * n + j] * Lf[(size_t)k * n + j];
                    if (!(sj > 0.0)) s.flag = 1;
                    else Lf[(size_t)j * n + j] = sqrt(sj);
                }
                __syncthreads();
                if (s.flag) break;
                const double ljj = Lf[(size_t)j * n + j];
                for (int i = j + 1 + tid; i < n; i += LM_THREADS) {
                    double t = Lf[(size_t)j * n + i];
                    for (int k = 0; k < j; ++k) t -= Lf[(size_t)k * n + i] * Lf[(size_t)k * n + j];
                    Lf[(size_t)j * n + i] = t / ljj;
                }
                __syncthreads();
            }
            if (s.flag) { terminate = true; break; }
            if (tid == 0) {
                double y[LM_MAXN];
                for (int i = 0; i < n; ++i) {
                    double t = (double)g[i];
                    for (int k = 0; k < i; ++k) t -= Lf[(size_t)k * n + i] * y[k];
                    y[i] = t / Lf[(size_t)i * n + i];
                }
                for (int i = n - 1; i >= 0; --i) {
                    double t = y[i];
                    for (int k = n - 1; k > i; --k) t -= Lf[(size_t)i * n + k] * y[k];
                    y[i] = t / Lf[(size_t)i * n + i];
                }
                for (int i = 0; i < n; ++i) d[i] = (float)(-y[i]);
                s.t = 1.0f;
            }
            __syncthreads();
            // line search: halve t until the objective decreases
            for (int inner = 0; inner < 100; ++inner) {
                const float t = s.t;
                if (t < 0.01f) { terminate = true; break; }
                for (int a = tid; a < n; a += LM_THREADS) zt[a] = z[a] + t * d[a];
                __syncthreads();
                lm_terms(m, xl, yl, bd, fs, cam, zt, false, s, F, nWx, nWy);
                if (tid == 0) {
                    s.ot = lm_objective(m, zt, tau, s);
                    s.flag = s.ot < s.obj;
                    s.t = t * 0.5f;
                }
                __syncthreads();
                if (s.flag) {
                    for (int a = tid; a < n; a += LM_THREADS) z[a] = zt[a];
                    __syncthreads();
                    break;
                }
            }
            __syncthreads();
        }
        __syncthreads();
    }
    for (int a = tid; a < K + 6; a += LM_THREADS) b.x[(size_t)f * m.KTP + a] = z[a];
    if (tid == 0) {
        if (success_out) success_out[f] = success;
        if (slack_out) slack_out[f] = z[nb];
        if (iters_out) iters_out[f] = iters;
    }
}

}  // namespace tdi
