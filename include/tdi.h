/*
 * tdi.h -- C ABI of the B200 implementation of 3DI's per-frame 3DMM fitting path.
 *
 * The path replaced is VideoFitter::fit_to_video_frame after the landmark initialisation
 * (src/lib/video_fitter.cu:432-648 of Computational-Psychiatry/3DI): blur of the target
 * crop, the light fit fit_3DMM_lambdas (src/lib/model_fitter.cu:981-1073), the shape fit
 * fit_3DMM_shape_rigid (model_fitter.cu:121-375), the optional two-stage repetition and
 * the expression finetune fit_3DMM_epsilon_finetune (model_fitter.cu:397-672), with the
 * renderer, derivative and solver calls they make (src/lib/renderer.cu,
 * derivative_computer.cu, logbarrier_initializer.cu, solver.h).
 *
 * Conventions: plain pointers and sizes, no CUDA or torch types (a stream is passed as
 * void*, NULL = the default stream); no global state; the caller owns inputs and outputs,
 * the library owns device scratch; errors are status codes (tdi_last_error() gives a
 * message). Images are 256x256 float crops stored column-major (pixel (x, y) at x*256+y),
 * as the reference stores them (video_fitter.cu:543-546).
 */
#ifndef TDI_H
#define TDI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t tdi_status;
#define TDI_OK 0
#define TDI_ERR_INVALID 1       /* bad argument */
#define TDI_ERR_CUDA 2          /* a CUDA call failed */
#define TDI_ERR_NOMEM 3         /* device or host allocation failed */
#define TDI_ERR_CAPACITY 4      /* more frames than the batch holds */

/* per-frame status bits of tdi_report.flags */
#define TDI_FLAG_RENDER_SKIPPED 1u   /* visible fragments outside [1000, 52000]: the reference
                                        skips the render (renderer.cu:669-677); frame stops */
#define TDI_FLAG_OUT_OF_DOMAIN 2u    /* an input the reference leaves undefined (fragments
                                        outside the crop or on its border, > 25,600 fragments) */
#define TDI_FLAG_NAN_DIRECTION 4u    /* NaN search direction (model_fitter.cu:206-213) */
#define TDI_FLAG_STUCK_NEG_TZ 8u     /* a trial with tau_z < 0 (model_fitter.cu:255-259) */
#define TDI_FLAG_CHOL_FAILED 16u     /* Cholesky factorisation failed (solver.h:87-92) */
#define TDI_FLAG_FAIL 32u            /* outer iterations <= NITERS_SUCCESS (model_fitter.cu:374) */
#define TDI_FLAG_OVERFLOW 64u        /* more than 32,768 fragments (tdi_raster_noalloc: more than capacity) */
#define TDI_FLAG_BAD_INDEX 128u      /* tdi_raster_noalloc: a triangle corner outside [0, n_vertices);
                                        that triangle is skipped */

typedef struct tdi_model tdi_model;
typedef struct tdi_batch tdi_batch;

/* Morphable model with the subject's identity applied (replaces the Renderer constructor's
 * file loading, renderer.cu:22-442, and the identity files of video_from_saved_identity.cu:
 * 141-150). Host arrays, copied to the device. */
typedef struct {
    int32_t n_vertices;          /* V */
    int32_t n_triangles;         /* T (the reference's 16-bit indices cap T at 65,535) */
    int32_t n_expr;              /* K, 79 for the GLOBAL79 basis */
    const float *mean;           /* [3][V] X0_mean, Y0_mean, Z0_mean (identity applied) */
    const float *expr_basis;     /* [V][3][K] rows of EX_79/EY_79/EZ_79.dat per vertex */
    const float *tex;            /* [V] albedo (tex_mu with the identity texture) */
    const int32_t *triangles;    /* [3][T] 0-based vertex ids (tl.dat columns minus 1) */
    const int32_t *landmarks;    /* [51] landmark vertex ids (config::LIS) */
    const float *eps_lb;         /* [K] expression bounds of the shape fit */
    const float *eps_ub;
    const float *eps_lb_finetune;/* [K] bounds of the expression finetune */
    const float *eps_ub_finetune;
} tdi_model_desc;

/* Frames of a batch; host arrays. The crop origin and face size follow the reference
 * (renderer.cu:580-598, funcs.cu:44-54) when x0y0 is NULL or face_size is NULL. */
typedef struct {
    int32_t n_frames;            /* F */
    const float *targets;        /* [F][65536] unblurred gray crops (the library blurs them) */
    const float *xl, *yl;        /* [F][51] landmarks in the rescaled frame */
    const float *bounds;         /* [F][4][51] lx, ly, ux, uy bound offsets in face sizes */
    const float *face_size;      /* [F] or NULL */
    const float *cam;            /* [F][4] phix, phiy, cx, cy of the rescaled camera */
    const int32_t *x0y0;         /* [F][2] crop origins, or NULL */
} tdi_frames;

/* Frames as the reference's video fitter receives them: 8-bit BGR images at their
 * original resolution, landmarks in original pixels, the original camera and each frame's
 * face size (video_fitter.cu:520-550, input_data.cu:32-53, camera.h:162-174). Host arrays. */
typedef struct {
    int32_t n_frames;            /* F */
    int32_t width, height;       /* size of every image */
    int64_t row_bytes;           /* bytes from one image row to the next (>= 3 width) */
    const uint8_t *bgr;          /* [F][height][row_bytes] B, G, R bytes per pixel */
    const float *xp, *yp;        /* [F][51] landmarks in image pixels */
    const float *bounds;         /* [F][4][51] lx, ly, ux, uy bound offsets in face sizes */
    const float *face_size;      /* [F] face size in image pixels */
    const float *cam;            /* [F][4] phix, phiy, cx, cy of the original camera */
    float ref_face_size;         /* REF_FACE_SIZE: frames are rescaled by ref_face_size / face_size */
    const float *ref_face_sizes; /* [F] per-frame reference sizes instead (the reference's scale
                                  * list, video_fitter.cu:271-280), or NULL */
} tdi_video_frames;

/* Orthographic pose initialisation of many frames (OrthographicInitializer::fit_model,
 * orthographic_initializer.cu:243-380): per frame a 7-parameter Gauss-Newton fit
 * x = (tau_x, tau_y, sigma_x, sigma_y, u1, u2, u3) of the scaled orthographic projection of
 * the model's landmark points p0L [3][51] (p0L_mat.dat) to the frame's centred landmarks
 * xl, yl [F][51], from the reference's start point. Outputs x [F][7], the yaw, pitch and roll
 * in degrees of the last trial rotation [F][3] (or NULL) and the outer iterations [F]
 * (or NULL). Host arrays; allocates its device buffers; synchronous. */
/* The subject's shape and albedo from identity and texture coefficients: the reference's
 * Renderer::compute_nonrigid_shape_identityonly and compute_texture (renderer.cu:866-883,941-951;
 * cublasSgemv there): mean[c][v] = mean0[c][v] + sum_k id_basis[c][v][k] alpha[k] (c = X, Y, Z)
 * and tex[v] = tex0[v] + sum_k tex_basis[v][k] beta[k], each sum a sequential FP32 fused
 * multiply-add chain over k from 0, added to the mean last (the reference's summation order is
 * the library's). Host arrays: mean0 [3][V], id_basis [3][V][n_id] (IX/IY/IZ.dat rows), alpha
 * [n_id], tex0 [V], tex_basis [V][n_tex] (TEX.dat rows), beta [n_tex]; outputs mean [3][V] and
 * tex [V], the inputs of tdi_model_create. n_id or n_tex may be 0 (a copy). Synchronous. */
tdi_status tdi_apply_identity(int32_t n_vertices, int32_t n_id, int32_t n_tex, const float *mean0,
                              const float *id_basis, const float *alpha, const float *tex0,
                              const float *tex_basis, const float *beta, float *mean, float *tex,
                              void *stream);

tdi_status tdi_orthographic_init(int32_t n_frames, const float *xl, const float *yl, const float *p0L,
                                 float *x_out, float *ypr_out, int32_t *iters_out, void *stream);

/* Configuration keys of the reference that the path reads (config.cu:350-541). */
typedef struct {
    int32_t max_iters_rigid;     /* outer GN iterations of the shape fit (100) */
    int32_t max_iters_finetune;  /* outer GN iterations of the finetune (100) */
    int32_t twostage_illum;      /* TWOSTAGE_ILLUM */
    int32_t finetune;            /* FINETUNE_EXPRESSIONS */
    int32_t niters_success;      /* NITERS_SUCCESS (6) */
    int32_t max_iters_lambda;    /* outer iterations of the light fit (10000) */
    float ref_face_size;         /* REF_FACE_SIZE */
    float taps[15];              /* Gaussian taps for KERNEL_SIGMA (video_fitter.cu:53-61) */
    int32_t normal_eq;           /* normal equations J^T J, J^T r (derivative_computer.cu:157-163):
                                  * 0 = FP64 sums in the oracle's fixed order (bit-exact);
                                  * 1 = split-BF16 products on the tensor cores, FP32
                                  *     accumulation per 256-fragment chunk (g stays exact).
                                  *     No counterpart in the reference (which uses
                                  *     cublasSgemm). */
    float damping;               /* lambda of the shape solve's damped Cholesky: the Gauss-Newton
                                  * system (H + lambda I) d = -g, lambda >= 0 added in FP64 to the
                                  * diagonal before the factorisation. 0 = the reference's undamped
                                  * solve (Solver::solve, solver.h:70-105). */
    int32_t host_rounds;         /* 0: the fitting rounds of a stage are replayed on the device from
                                  * CUDA graphs of 16 rounds, the host reading the active-frame count
                                  * once per replay; 1: the host launches every round and reads the
                                  * count after each (the same kernels and results). */
    int32_t vertex_stage;        /* basis x coefficients of the vertex stage (renderer.cu:806-861):
                                  * 0 = FP32 fused multiply-add chains in the oracle's order
                                  * (bit-exact); 1 = split-BF16 products on the tensor cores with
                                  * FP32 accumulation (at most 80 expression components). Applies
                                  * to tdi_batch_fit and tdi_batch_evaluate. */
} tdi_fit_config;

typedef struct {
    uint32_t flags;              /* TDI_FLAG_* */
    int32_t n_fragments;         /* visible fragments of the last render */
    int32_t iters_rigid;         /* num_outer_iters summed over the shape fits */
    int32_t iters_finetune;
    int32_t iters_lambda;        /* outer light-fit iterations */
    int32_t renders;             /* rasterisations */
    float objective;             /* last accepted objective */
} tdi_report;

const char *tdi_last_error(void);

/* Model: replaces the Renderer/Logbarrier_Initializer model loading
 * (renderer.cu:22-442, logbarrier_initializer.cu:30-440). */
tdi_status tdi_model_create(const tdi_model_desc *desc, tdi_model **out);
tdi_status tdi_model_destroy(tdi_model *m);

/* Batch: device working set for up to max_frames frames fitted together (replaces the
 * per-VideoFitter Optimizer/OptimizationVariables/Solver allocations, Optimizer.h:24-361). */
tdi_status tdi_batch_create(tdi_model *m, int32_t max_frames, tdi_batch **out);
tdi_status tdi_batch_destroy(tdi_batch *b);

/* Upload frames and blur the targets (video_fitter.cu:537-550). Synchronous. */
tdi_status tdi_batch_set_frames(tdi_batch *b, const tdi_frames *frames, void *stream);
/* Upload raw video frames and form their crops on the device: the reference's
 * get_resized_frame + crop (input_data.cu:43-53, video_fitter.cu:537-550; OpenCV's
 * BGR2GRAY, /255, INTER_LINEAR resize by ref_face_size / face_size, zero border, 256x256
 * crop at the origin from the rescaled landmarks), its get_resized_landmarks and
 * update_camera. Replaces tdi_batch_set_frames for callers holding decoded video frames.
 * Synchronous. */
tdi_status tdi_batch_set_video_frames(tdi_batch *b, const tdi_video_frames *frames, void *stream);
/* Upload states: x [F][K+6] (epsilon, tau_x, tau_y, tau_z, u1, u2, u3), lam [F][3],
 * light intensity L [F]. x may be NULL: the states on the device stay (after
 * tdi_batch_landmark_init); only the light is set. Synchronous. */
tdi_status tdi_batch_set_state(tdi_batch *b, const float *x, const float *lam, const float *L,
                               void *stream);
/* Landmark initialisation of the batch's frames (after tdi_batch_set_frames or
 * tdi_batch_set_video_frames), what VideoFitter::fit_to_video_frame runs before the image fit
 * (video_fitter.cu:456-500): per frame the orthographic pose fit to the landmarks with the
 * landmark points p0L [3][51] (p0L_mat.dat; tdi_orthographic_init's method, refitted from the
 * Euler angles when it ends mirrored), its perspective start, the smallest feasible slack and
 * the log-barrier fit of pose and expressions to the landmark boxes with a slack variable
 * (Logbarrier_Initializer::initialize_with_orthographic_t, set_minimal_slack, fit_model;
 * logbarrier_initializer.cu:1041-1269,1862-1918). The expression bounds are the model's shape-fit
 * bounds; the landmark 3D points are the model's mean and expression basis at its landmarks.
 * Writes the batch's states on the device (the start of tdi_batch_fit; set the light with
 * tdi_batch_set_state(b, NULL, lam, L)); per frame (host arrays, each may be NULL): success [F]
 * (1 when the slack went below -0.01, the reference's fit_success), the final slack [F] and the
 * Newton iterations [F]. Synchronous. */
tdi_status tdi_batch_landmark_init(tdi_batch *b, const float *p0L, int32_t *success, float *slack,
                                   int32_t *iters, void *stream);

/* Fit every frame of the batch on the device (asynchronous on the stream apart from one
 * 4-byte read-back per round). Replaces fit_to_video_frame's fitting calls. */
tdi_status tdi_batch_fit(tdi_batch *b, const tdi_fit_config *cfg, void *stream);
/* Download states and reports. Synchronous. */
tdi_status tdi_batch_get_state(tdi_batch *b, float *x, float *lam, tdi_report *rep, void *stream);

/* All of the above for host buffers: upload, fit, download (x and lam are in/out). */
tdi_status tdi_fit_frames(tdi_batch *b, const tdi_frames *frames, const tdi_fit_config *cfg,
                          float *x, float *lam, const float *L, tdi_report *rep, void *stream);

/* One full evaluation of every frame at its current state -- what one outer iteration of
 * fit_3DMM_shape_rigid computes before its line search (get_obj_hessian_and_gradient_multiframe
 * and Solver::solve, model_fitter.cu:21-116,179-201) -- kept on the device for
 * tdi_batch_read. finetune_bounds selects the finetune expression bounds. */
tdi_status tdi_batch_evaluate(tdi_batch *b, const tdi_fit_config *cfg, int32_t finetune_bounds,
                              void *stream);

/* Read one frame's working set after tdi_batch_evaluate or tdi_batch_raster. what:
 *  0 fragments   int32 [N][4]: pixel | owner<<31, triangle, float bits of alpha, beta
 *  1 neighbours  int32 [4][N]: kl, kr, ka, kb
 *  2 gradients   float [5][N]: gx, gy, h, target gx/|g|, target gy/|g|
 *  3 jacobian    float [N][K+6]
 *  4 normal eq.  float [K+6][K+6] H, then [K+6] g, then [K+6] direction d
 *  5 scalars     double [4]: correlation, barrier objective, objective, face check
 *  6 geometry    float [6][V]: X0, Y0, Z0, xp, yp, camera Z
 *  7 crop        float [65536]: the unblurred crop, x-major (after set_frames / set_video_frames)
 *  8 frame data  float [109]: xl [51], yl [51], camera [4], face size, crop origin x0, y0
 * Returns the number of elements written through *count. Synchronous. */
tdi_status tdi_batch_read(tdi_batch *b, int32_t frame, int32_t what, void *dst, int64_t capacity,
                          int64_t *count);

/* Visibility of given projections (the reference's get_pixels_to_render, keep_only_minZ and
 * remove_if, funcs.cu:900-1029, renderer.cu:650-680) for one frame slot of the batch: xp, yp
 * and camera Z per vertex, crop origin. Results are read with tdi_batch_read(what=0).
 * Synchronous; returns the fragment count through *n_out. */
tdi_status tdi_batch_raster(tdi_batch *b, int32_t frame, const float *xp, const float *yp,
                            const float *zc, int32_t x0, int32_t y0, int32_t *n_out,
                            uint32_t *flags_out);

/* Render every frame of the batch at its current state, as Renderer::render does before
 * the blur (renderer.cu:635-696): unblurred image [F][65536] and the triangle that owns each
 * pixel [F][65536] (-1 where nothing is drawn). Either output may be NULL. Synchronous. */
tdi_status tdi_batch_render(tdi_batch *b, float *images, int32_t *tri_map, void *stream);

/* Differentiable render loss of every frame of the batch (after tdi_batch_set_frames), for the
 * torch.autograd.Function of the Python package; no counterpart in the reference, whose fit uses
 * the warp-only Jacobian contracted with the residual (derivative_computer.cu:157-164).
 * loss[f] = -sum_n (gxn_n gxsn_n + gyn_n gysn_n): the negated correlation of the normalised
 * gradients of the blurred render and target at the frame's fragments (funcs.cu:842-897), the
 * image term the shape fit minimises (scaled there by tau_img = 25). The fragments (triangle and
 * pixel of every sample, the owner of every pixel) come from the library's raster at x and are
 * then held; barycentrics, geometry, shading, blur and gradients are FP64 functions of
 * (epsilon, tau, u, lambda, L), so the loss is smooth in them. DEVICE pointers: x [F][K+6],
 * lam [F][3], L [F] (float), loss [F] (double); cfg supplies the blur taps. Asynchronous on the
 * stream except one 8-byte read-back. */
tdi_status tdi_batch_loss(tdi_batch *b, const tdi_fit_config *cfg, const float *x, const float *lam,
                          const float *L, double *loss, void *stream);
/* Gradient of sum_f gloss[f] loss[f] by the hand-written adjoint (raster and FP64 forward
 * recomputed, nothing stored between the calls): gx [F][K+6] (epsilon, tau, u), glam [F][3] and
 * gL [F] (double, DEVICE pointers; glam, gL may be NULL). */
tdi_status tdi_batch_loss_backward(tdi_batch *b, const tdi_fit_config *cfg, const float *x, const float *lam,
                                   const float *L, const double *gloss, double *gx, double *glam, double *gL,
                                   void *stream);

/* Kernels launched by this batch since it was created (each a hand-written CUDA kernel). */
tdi_status tdi_batch_launches(tdi_batch *b, int64_t *launches);

/* Live timing of one kernel for roofline reports: while kernel_id != 0, every launch of that
 * kernel is bracketed by CUDA events on its stream and the frames it processed are counted
 * on the device. kernel_id: 1 vertex stage, 2 visibility depth pass, 3 render, 4 neighbour
 * maps, 5 Jacobian rows, 6 normal equations, 7 barrier terms, 8 Cholesky, 9 visibility
 * resolve (fragment list). profile_read returns the launches, their summed milliseconds and
 * the frames they processed since profile() was called (synchronises). */
tdi_status tdi_batch_profile(tdi_batch *b, int32_t kernel_id);
tdi_status tdi_batch_profile_read(tdi_batch *b, int64_t *launches, double *total_ms,
                                  int64_t *frames);

/* Visibility of one frame for callers that cannot allocate device memory (no counterpart in
 * 3DI, which allocates all of its working memory up front). Same result as tdi_batch_raster
 * for the same projections: device arrays xp, yp, camera Z [n_vertices], triangles
 * [3][n_triangles] (0-based), crop origin; output: fragments int32 [capacity][4] (pixel |
 * owner<<31, triangle, float bits of alpha, beta) in slot order, *count (device int32, the
 * number written, at most capacity; TDI_FLAG_OVERFLOW when more survived) and *flags (device
 * uint32, TDI_FLAG_*). A triangle with a corner outside [0, n_vertices) is skipped on the
 * device before any vertex is read (TDI_FLAG_BAD_INDEX). Calls no allocator: its working
 * memory is a fixed 640 KiB array in the library's device image, held on every device that
 * loads the library until the process exits. At most 131,072 triangles (TDI_ERR_CAPACITY
 * otherwise). Calls share that array: calls that overlap on the GPU race; serialise them on
 * one stream. Every call looks the array up (cudaGetSymbolAddress, no allocation) with the
 * caller's device current; the first call on a device also loads the library's device code
 * there, so make it before any stream capture. Asynchronous on the stream. */
tdi_status tdi_raster_noalloc(const float *xp, const float *yp, const float *zc,
                              const int32_t *triangles, int32_t n_vertices, int32_t n_triangles,
                              int32_t x0, int32_t y0, int32_t *fragments, int32_t capacity,
                              int32_t *count, uint32_t *flags, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TDI_H */
