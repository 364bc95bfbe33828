/*
 * CPU oracle for the 3DI per-frame fitting path. TEST INFRASTRUCTURE ONLY: the checker
 * that tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg call; the product
 * (3di_b200/) never links or calls it.
 *
 * Built twice from tdi_oracle.c:
 *   libtdi_oracle_f32.so  REAL = float: the reference's FP32 arithmetic, operation by
 *                         operation, as the reference sources would compute it without
 *                         FMA contraction (nvcc -fmad=false / gcc -ffp-contract=off).
 *   libtdi_oracle_f64.so  REAL = double: the FP64 oracle. Visibility (which fragments are
 *                         drawn) is decided in FP32 on FP32-rounded projections in both
 *                         builds, so the two share their discrete structure.
 *
 * Parity status: the reference ships no tests, golden vectors or fixtures for this path, so
 * the restatement is pinned to the reference itself. ref.mk builds its hot-path CUDA sources
 * as they lie into _ref/, with stand-in headers for the OpenCV display helpers that the path
 * never calls. tests/test_ref_pinning.py compares the two stage by stage on a B200. Every
 * function cites the reference file:line it restates.
 *
 * Layouts (shared with the product's C ABI, include/tdi.h):
 *   images     256x256 float, column-major: pixel (x, y) at x*256 + y
 *   mean       [3][V]      planes X, Y, Z
 *   E          [V][3][K]   expression basis rows per vertex and coordinate
 *   tl         [3][T]      0-based vertex ids, plane r holds column r of tl.dat
 *   state x    [K+6]       epsilon[K], tau_x, tau_y, tau_z, u1, u2, u3
 *   bounds     [4][51]     lx, ly, ux, uy as fractions of the face size
 */
#ifndef TDI_ORACLE_H
#define TDI_ORACLE_H
#include <stdint.h>

#define O_NL 51
#define O_DIM 256
#define O_NPIX 65536
#define O_NTMP 4
#define O_NTAPS 15

typedef struct {
    int32_t V, T, K;
    const float *mean;
    const float *E;
    const float *tex;
    const int32_t *tl;
    const int32_t *lis;
    const float *eps_lb, *eps_ub, *eps_lb_ft, *eps_ub_ft;
} o_model;

typedef struct {
    const float *target;       /* unblurred crop */
    const float *xl, *yl;      /* [51] landmarks in the rescaled frame */
    const float *bounds;       /* [4][51] */
    float face_size;
    float phix, phiy, cx, cy;
    int32_t x0, y0;
} o_frame;

typedef struct {
    int32_t max_iters_rigid;     /* outer GN iterations of fit_3DMM_shape_rigid (100) */
    int32_t max_iters_finetune;  /* outer GN iterations of fit_3DMM_epsilon_finetune (100) */
    int32_t twostage_illum;      /* TWOSTAGE_ILLUM */
    int32_t finetune;            /* FINETUNE_EXPRESSIONS */
    int32_t niters_success;      /* NITERS_SUCCESS (6) */
    int32_t max_iters_lambda;    /* outer iterations of fit_3DMM_lambdas (10000) */
    float ref_face_size;         /* REF_FACE_SIZE */
    float taps[O_NTAPS];         /* Gaussian blur taps */
    float damping;               /* lambda of the damped shape solve (H + lambda I); 0 = undamped */
} o_config;

/* frame status bits */
#define O_FLAG_RENDER_SKIPPED   1u   /* N outside [1000, 52000] (renderer.cu:669-677) */
#define O_FLAG_OUT_OF_DOMAIN    2u   /* a case the reference leaves undefined */
#define O_FLAG_NAN_DIRECTION    4u   /* NaN search direction (model_fitter.cu:206-213) */
#define O_FLAG_STUCK_NEG_TZ     8u   /* trial with tau_z < 0 (model_fitter.cu:255-259) */
#define O_FLAG_CHOL_FAILED     16u   /* potrf failure (solver.h:87-92) */
#define O_FLAG_FAIL            32u   /* fit not successful (outer iterations <= NITERS_SUCCESS) */

typedef struct {
    uint32_t flags;
    int32_t n_fragments;         /* N of the last full render */
    int32_t iters_rigid;         /* num_outer_iters summed over shape fits */
    int32_t iters_finetune;
    int32_t iters_lambda;        /* outer illumination iterations */
    int32_t renders;             /* full + trial renders */
    float objective;             /* last accepted objective */
} o_report;

#endif
