/*
 * wos_b200.h -- C ABI of the B200 walk-on-spheres library (libwos_b200.so).
 *
 * This is the drop-in boundary for the hot path of diff-wos.  It replaces the
 * reference's pybind module `wos_ext` (src/python/main.cpp:9-17,
 * src/python/scene.cu:10-88, src/python/wos.cu:5-25), whose arguments were
 * Dr.Jit CUDA arrays, with plain pointers and sizes:
 *
 *   - every array argument is a pointer to DEVICE memory of the current CUDA
 *     device (for example a torch CUDA tensor's data_ptr()), C-contiguous;
 *     points and vertices are n x dim float32, faces are nF x dim int32;
 *   - every call takes the cudaStream_t it runs on and is asynchronous on it,
 *     except wos_scene_create / wos_scene_update_vertices, which return
 *     after the scene is built;
 *   - every call returns 0 on success or a negative WOS_ERR_* code, and
 *     wos_last_error_string() describes the last failure of this thread;
 *   - a scene handle is immutable between wos_scene_update_* calls and may be
 *     used by concurrent launches on different streams.
 *
 * Randomness is counter based: a walk's random numbers are Philox-4x32-10 of
 * (seed; point index, walk index, step, role), so results do not depend on
 * launch shape, scheduling or how many walks run per call.
 */
#ifndef WOS_B200_H
#define WOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define WOS_API __attribute__((visibility("default")))
#else
#define WOS_API
#endif

typedef struct CUstream_st *wos_stream_t; /* == cudaStream_t */
typedef struct wos_scene_s *wos_scene_t;

enum {
    WOS_OK = 0,
    WOS_ERR_INVALID_ARGUMENT = -1,
    WOS_ERR_CUDA = -2,
    WOS_ERR_EMPTY_SCENE = -3,
    WOS_ERR_UNSUPPORTED = -4,
    WOS_ERR_WORKSPACE = -5,
};

/* Device status bits OR-ed by kernels (wos_device_status). */
enum {
    WOS_STATUS_STACK_OVERFLOW = 1,
    WOS_STATUS_BAD_PRIM = 2,
    WOS_STATUS_NONFINITE = 4,
    WOS_STATUS_QUEUE_LIMIT = 8,
};

/* Solver settings.  Mirrors wos_ext.WoS / WoS3D(nwalks, nsteps=32,
 * epsilon=1e-3, double_sided=False, prevent_fd_artifacts=False,
 * use_IS_for_greens) (src/python/wos.cu:9-12) plus:
 *   include_source       add the interior source term to each walk's value
 *                        (WoSWithSourceCUDA.single_walk,
 *                        wos/wos_with_source.py:257-265); 0 gives the
 *                        WoSCUDA value (wos/wos.py:171-179);
 *   project_unterminated 0: a walk that reaches nsteps is invalid and scores 0
 *                        (include/wos.cuh:144); 1: it is projected to its
 *                        closest boundary point (the Dr.Jit walk, wos/wos.py:43);
 *   use_bvh              1: LBVH nearest queries, 0: brute force
 *                        (include/scene.cuh:150-154);
 *   walk_offset          first walk index (the sampler's position);
 *   seed                 64-bit Philox key;
 *   jitter               per-axis extent of the start-point jitter: walk w of
 *                        point i starts at P[i] + (u - 1/2) * jitter with u
 *                        uniform per axis from the walk's own random numbers
 *                        (pixel sampling of Solver.walk_detector,
 *                        wos/solver.py:67-84, wos/scene.py:33-39); zeros
 *                        start every walk at P[i]. */
typedef struct wos_params {
    int32_t nwalks;
    int32_t nsteps;
    float epsilon;
    int32_t double_sided;
    int32_t prevent_fd_artifacts;
    int32_t use_IS_for_greens;
    int32_t include_source;
    int32_t project_unterminated;
    int32_t use_bvh;
    uint32_t walk_offset;
    uint64_t seed;
    float jitter[3];
} wos_params;

/* Settings of the differential estimator (OursCUDA / Ours3D,
 * wos/wos_grad.py:113-151, wos/wos_grad_3d.py:104-137):
 *   epsilon2                    shell width of the walks on the inscribed ball;
 *   clamping                    angle clamp of the off-centred Poisson kernel;
 *   control_variates            subtract u at the boundary point (wos/wos.py:103);
 *   source_in_normal_derivative use the source-aware normal derivative
 *                               (wos/wos_with_source.py:154-232) when the
 *                               scene has a source (2D);
 *   ball_epsilon                lower bound of the inscribed-ball bisection
 *                               (include/scene.cuh:225, default 1e-3);
 *   want_dV / want_dg / want_dsrc  which gradients to accumulate. */
typedef struct wos_adjoint_params {
    float epsilon2;
    float clamping;
    int32_t control_variates;
    int32_t source_in_normal_derivative;
    float ball_epsilon;
    int32_t want_dV;
    int32_t want_dg;
    int32_t want_dsrc;
} wos_adjoint_params;

typedef struct wos_scene_info {
    int32_t dim, n_vertices, n_faces, n_nodes, bvh_depth, source_type;
    float aabb_min[3], aabb_max[3];
    float source_params[5];
} wos_scene_info;

/* Library version (major * 10000 + minor * 100 + patch). */
WOS_API int wos_version(void);

/* Message of this thread's last failing call ("" if none). */
WOS_API const char *wos_last_error_string(void);

/* Device status word of the current device; reset != 0 clears it.  Reading it
 * synchronises the device. */
WOS_API int wos_device_status(int reset, int32_t *out);

/* ---------------------------------------------------------------- scenes */

/* Build a scene: copies vertices V (nV x dim), faces F (nF x dim, CCW
 * polylines / outward-oriented triangles), Dirichlet values g (nV); computes
 * vertex normals, the AABB and the LBVH.  source_params is a HOST array of 5
 * floats (NULL for none).  Replaces wos_ext.Scene(vertices, indices, values,
 * use_bvh[, source_type, source_params]) / Scene3D (src/python/scene.cu:28-83,
 * include/scene.cuh:330-453).  Returns after the build completes. */
WOS_API int wos_scene_create(int dim, const float *V, int nV, const int *F, int nF, const float *g, int source_type,
                     const float *source_params, wos_stream_t stream, wos_scene_t *out);

/* Free a scene (stream-ordered on `stream`). */
WOS_API int wos_scene_destroy(wos_scene_t scene, wos_stream_t stream);

/* Replace the Dirichlet values (nV floats, device).  The scene's `values`
 * field (src/python/scene.cu:38). */
WOS_API int wos_scene_update_values(wos_scene_t scene, const float *g, wos_stream_t stream);

/* Replace vertex positions (nV x dim, device) and rebuild normals, AABB and
 * LBVH; returns after the rebuild.  The scene's device buffers stay where they
 * are (the trees are refilled in place), so batch plans and launches that hold
 * the scene keep reading live memory; kernels still running on another stream
 * race with the rebuild and must be ordered before it by the caller. */
WOS_API int wos_scene_update_vertices(wos_scene_t scene, const float *V, wos_stream_t stream);

/* Set the analytic source (include/scene.cuh:270-301): type 0 none,
 * 1 Gaussian (mu_x, mu_y, sigma_x, sigma_y, A), 2 sinusoid
 * (A, B, C, amplitude, offset) = amplitude * sin(A x + B y + C) + offset.
 * params is a HOST array of 5 floats.  The walk solves -Lap u = f. */
WOS_API int wos_scene_set_source(wos_scene_t scene, int source_type, const float *params);

WOS_API int wos_scene_get_info(wos_scene_t scene, wos_scene_info *out);

/* Copy the vertex normals (nV x dim, device) into out (device). */
WOS_API int wos_scene_get_normals(wos_scene_t scene, float *out, wos_stream_t stream);

/* ---------------------------------------------------------------- queries */

/* Closest boundary point of n points P (n x dim): Scene.closest_point_preliminary
 * (include/scene.cuh:102-146), closest_point (:180-223) and sdf (:148-178).
 * Any output may be NULL.  prim: nearest primitive (ties to the lowest index);
 * dist: unsigned distance; t_or_uv: n x 2 (2D: (t, 0), 3D: (w_b, w_c));
 * pt, normal: n x dim (normal oriented towards the query point);
 * sdf: signed distance (negative inside); inside: 1 if the point is inside
 * (the test that gates a walk). */
WOS_API int wos_closest_point(wos_scene_t scene, const float *P, int n, int use_bvh, int32_t *prim, float *dist,
                      float *t_or_uv, float *pt, float *normal, float *sdf, uint8_t *inside, wos_stream_t stream);

/* Scene.sdf (include/scene.cuh:148-178): signed distance of n points P
 * (n x dim) to the boundary, negative inside; the sdf output of
 * wos_closest_point alone. */
WOS_API int wos_sdf(wos_scene_t scene, const float *P, int n, int use_bvh, float *sdf, wos_stream_t stream);

/* Scene.largest_inscribed_ball(its, epsilon) (include/scene.cuh:225-249,
 * :659-704): 10-step bisection of the ball tangent at boundary point pt with
 * inward normal `normal`; R = 0 where valid == 0. */
WOS_API int wos_largest_inscribed_ball(wos_scene_t scene, const uint8_t *valid, const float *pt, const float *normal, int n,
                               float epsilon, int use_bvh, float *R, wos_stream_t stream);

/* ---------------------------------------------------------------- walks */

/* One walk per point with walk index p->walk_offset; the record of
 * WoS.single_walk(p, scene, sampler) (include/wos.cuh:374-533).  valid: n;
 * pt, normal: n x dim; t_or_uv: n x 2; prim: n (-1 if invalid); contrib: n
 * (source term).  Any output except valid may be NULL. */
WOS_API int wos_walk_records(wos_scene_t scene, const float *P, int n, const wos_params *p, uint8_t *valid, float *pt,
                     float *normal, float *t_or_uv, int32_t *prim, float *contrib, wos_stream_t stream);

/* Per-walk values: values[i * nwalks + w] = value of walk w of point i
 * (0 for an invalid walk).  steps (may be NULL): steps per walk. */
WOS_API int wos_walk_values(wos_scene_t scene, const float *P, int n, const wos_params *p, float *values, int32_t *steps,
                    wos_stream_t stream);

/* Workspace bytes for wos_solve with n points. */
WOS_API size_t wos_solve_workspace_size(int n, const wos_params *p);

/* Solver.walk / solve (wos/solver.py:41-65): per-point mean over nwalks
 * walks and the sample variance of the per-walk values, reduced in FP64
 * with compensated sums.  var may be NULL.  workspace may be NULL (then it
 * is allocated stream-ordered) or point to wos_solve_workspace_size bytes of
 * device memory. */
WOS_API int wos_solve(wos_scene_t scene, const float *P, int n, const wos_params *p, double *mean, double *var,
              void *workspace, size_t workspace_bytes, wos_stream_t stream);

/* ---------------------------------------------------------------- gradients */

/* WoS.normal_derivative(its, scene, sampler, clamping, control_variates)
 * (wos/wos.py:59-107; with source wos/wos_with_source.py:154-232; 3D
 * wos/wos3d.py:97-135): one estimate per record, returned as grad * n_out
 * (n x dim).  Records as from wos_walk_records; walk index p->walk_offset. */
WOS_API int wos_normal_derivative(wos_scene_t scene, const uint8_t *valid, const float *pt, const float *normal,
                          const float *t_or_uv, const int32_t *prim, int n, const wos_params *p,
                          const wos_adjoint_params *a, float *out, wos_stream_t stream);

/* wos_normal_derivative on balls of given radii R (n floats, device) instead
 * of the largest inscribed ball: WoS.normal_derivative(..., override_R=R)
 * (wos/wos.py:59-107, override_R at :71-74; wos/wos_with_source.py:167-172).
 * The ball of record i is centred at pt - n_out R[i]. */
WOS_API int wos_normal_derivative_radius(wos_scene_t scene, const uint8_t *valid, const float *pt, const float *normal,
                                         const float *t_or_uv, const int32_t *prim, const float *R, int n,
                                         const wos_params *p, const wos_adjoint_params *a, float *out,
                                         wos_stream_t stream);

/* Workspace bytes for wos_adjoint on this scene. */
WOS_API size_t wos_adjoint_workspace_size(wos_scene_t scene);

/* Reverse-mode derivative of the per-point means of wos_solve with respect
 * to vertex positions (dV, nV x dim), Dirichlet values (dg, nV) and source
 * parameters (dsrc, 5): out += sum_i dLdu[i] d mean_i / d theta.  This is
 * CustomSolver.backward with OursCUDA / Ours3D (wos/solver.py:109-114,
 * wos/wos_grad.py:130-151, wos/wos_grad_3d.py:117-137) plus the gathers the
 * forward attaches (wos/scene.py:353-357, wos/wos_with_source.py:89-90).
 * Walks are recomputed from their Philox counters (same seed as the forward
 * solve gives common random numbers).  Outputs are float32 device arrays that
 * are ADDED to; any may be NULL when the matching want_* is 0. */
WOS_API int wos_adjoint(wos_scene_t scene, const float *P, int n, const wos_params *p, const wos_adjoint_params *a,
                const float *dLdu, float *dV, float *dg, float *dsrc, void *workspace, size_t workspace_bytes,
                wos_stream_t stream);

/* ---------------------------------------------------------------- fused */

/* Bytes of one per-walk boundary record (8 in 2D, 16 in 3D). */
WOS_API size_t wos_walk_record_bytes(int dim);

/* wos_solve that also stores each walk's boundary record into `records`
 * (n * nwalks * wos_walk_record_bytes(dim) bytes, device) and, if dcontrib is
 * not NULL, the derivative of its source term with respect to the 5 source
 * parameters (n * nwalks * 5 floats), for a later wos_adjoint_records. */
WOS_API int wos_solve_records(wos_scene_t scene, const float *P, int n, const wos_params *p, double *mean, double *var,
                              void *records, float *dcontrib, void *workspace, size_t workspace_bytes,
                              wos_stream_t stream);

/* wos_adjoint that starts each sample from the record its primal walk left in
 * wos_solve_records (same P, n and params) instead of walking it again --
 * the reference recomputes the primal walk from the seed
 * (wos/solver.py:109-114); the records make that recomputation unnecessary
 * and the result is the same.  Its workspace is wos_adjoint_workspace_size
 * bytes; given wos_adjoint_records_workspace_size bytes (or NULL) it also runs
 * the samples in boundary-primitive order (wos_set_sample_order). */
WOS_API size_t wos_adjoint_records_workspace_size(wos_scene_t scene, int n, const wos_params *p);
WOS_API int wos_adjoint_records(wos_scene_t scene, const float *P, int n, const wos_params *p,
                                const wos_adjoint_params *a, const float *dLdu, const void *records,
                                const float *dcontrib, float *dV, float *dg, float *dsrc, void *workspace,
                                size_t workspace_bytes, wos_stream_t stream);

WOS_API size_t wos_solve_adjoint_workspace_size(wos_scene_t scene, int n, const wos_params *p,
                                                const wos_adjoint_params *a);

/* Fused forward + adjoint step for a pointwise loss of the per-point means:
 * wos_solve_records, the loss and dL/du, then wos_adjoint_records, in one
 * call (one stream, no host round trip).  loss_kind 1: L = mean(u^2);
 * 2: L = mean((u - target)^2) with target = target_or_dLdu (n floats);
 * 0: dL/du given in target_or_dLdu.  loss (1 double, may be NULL) receives L
 * (kinds 1, 2).  Gradients are added to dV / dg / dsrc (float32). */
WOS_API int wos_solve_adjoint(wos_scene_t scene, const float *P, int n, const wos_params *p,
                              const wos_adjoint_params *a, int loss_kind, const float *target_or_dLdu, double *mean,
                              double *var, double *loss, float *dV, float *dg, float *dsrc, void *workspace,
                              size_t workspace_bytes, wos_stream_t stream);

/* Workspace of wos_solve_tangent. */
WOS_API size_t wos_solve_tangent_workspace_size(wos_scene_t scene, int n, const wos_params *p,
                                                const wos_adjoint_params *a);

/* Fused forward solve + forward-mode derivative of the per-point means along
 * a direction of the scene: dV_dir (nV x dim), dg_dir (nV) and dsrc_dir (5),
 * each may be NULL (no motion of that input; also skipped unless the
 * matching want_* flag of `a` is set).  tangent[i] (and tangent_var[i], may
 * be NULL) receive the mean (and sample variance) over point i's walks of
 * each walk's directional derivative: the boundary-shape term
 * -(grad_n u + grad_t g) . dx with dx the motion of the walk's boundary point,
 * plus the Dirichlet gather and the source term.  This is what the
 * reference's forward-mode renderings compute (dr.forward_to on a scene
 * parameter, diff_solve/runner.py:75-109); the estimator is the same as
 * wos_solve_adjoint's, so tangent summed against weights equals the adjoint
 * of that weighting dotted with the direction. */
WOS_API int wos_solve_tangent(wos_scene_t scene, const float *P, int n, const wos_params *p,
                              const wos_adjoint_params *a, const float *dV_dir, const float *dg_dir,
                              const float *dsrc_dir, double *mean, double *var, double *tangent, double *tangent_var,
                              void *workspace, size_t workspace_bytes, wos_stream_t stream);

/* Workspace of wos_soft_walk. */
WOS_API size_t wos_soft_walk_workspace_size(int n, const wos_params *p);

/* The soft-edge walk of the reference's Baseline / Baseline3D
 * (wos/wos.py:158-187, wos/wos_grad_3d.py:24-57): every walk takes exactly
 * p->nsteps steps (nsteps >= 1), each adding beta (1 - w) g(closest point)
 * with w = min(d, epsilon) / epsilon, then beta *= w; p->epsilon is the
 * soft-edge width.  mean / var: per-point mean and variance of the walk
 * values.  Forward mode: when `tangent` is given, the per-point mean (and
 * variance) of each walk's derivative along dV_dir (nV x dim) and dg_dir
 * (nV), either may be NULL: the motion of every step's distance, weight,
 * position and boundary value is carried through the walk (the reference
 * differentiates the same walk with Dr.Jit). */
WOS_API int wos_soft_walk(wos_scene_t scene, const float *P, int n, const wos_params *p, const float *dV_dir,
                          const float *dg_dir, double *mean, double *var, double *tangent, double *tangent_var,
                          void *workspace, size_t workspace_bytes, wos_stream_t stream);

/* Reverse mode of wos_soft_walk (the Baseline / Baseline3D walks are fully
 * attached in the reference, wos/wos.py:170-187, wos/wos_grad_3d.py:39-57, so
 * Dr.Jit differentiates them in either mode): dV (nV x dim) and dg (nV),
 * float32 device arrays that are ADDED to (either may be NULL), receive
 * sum_i dLdu[i] d mean_i / d(vertices, values) over the same walks as
 * wos_soft_walk with the same params.  Each walk is repeated from its Philox
 * counters and its per-step positions are kept in scratch memory allocated
 * stream-ordered (at most 256 MB at a time; walks are processed in chunks). */
WOS_API int wos_soft_walk_adjoint(wos_scene_t scene, const float *P, int n, const wos_params *p, const float *dLdu,
                                  float *dV, float *dg, wos_stream_t stream);

/* A detector: res[0] x res[1] pixels over [vmin, vmax] in scene axes
 * (axis_u, axis_v); in 3D a slab |x[slab_axis] - slab_center| <
 * slab_half_width (slab_axis -1 in 2D); size = its area (2D) or slab volume
 * (3D) (Detector / Detector3D / Detector3DY, wos/scene.py:9-42,
 * wos/scene3d.py:9-85).  Pixel of a point: u = (x[axis_u] - vmin[0]) /
 * (vmax[0] - vmin[0]) * res[0] + 0.5 truncated, likewise v, index
 * u + (res[1] - v) * res[0] (the reference's Detector.index); points whose
 * index falls outside the image are dropped. */
typedef struct wos_detector {
    float vmin[2];
    float vmax[2];
    int32_t res[2];
    int32_t axis_u, axis_v;
    int32_t slab_axis;
    float slab_center, slab_half_width;
    float size;
    int32_t flags; /* WOS_DETECTOR_* bits */
} wos_detector;

/* wos_detector.flags: divide a 3D sample's pmf by |ab x ac| as the
 * reference's Scene3D.sample_boundary does (wos/scene3d.py:251, :262), which
 * is twice the triangle's area and doubles the 3D boundary term; without it
 * the pdf is the correct 1 / (total area).  2D is the same either way. */
#define WOS_DETECTOR_REFERENCE_AREA_PDF 1

/* Image-space boundary term of the shape derivative (WoSBoundary,
 * wos/wos_boundary.py:11-31): res[0] * res[1] * nwalks boundary points drawn
 * uniformly by length (2D) or area (3D) with Philox(seed); each contributes
 * -g(x) (n . dx) / pdf / (size * nwalks) to its pixel, n the primitive's
 * normal (-ab.y, ab.x)/|ab| in 2D and -(ab x ac)/|ab x ac| in 3D, dx the
 * motion of the sampled point.  Forward mode: dV_dir (nV x dim) and
 * image_tangent (npixels doubles, added to).  Reverse mode: dLdI (npixels)
 * and dV (nV x dim floats, added to).  Either pair may be NULL.  The 3D pdf
 * is 1 / (total area) unless det->flags has WOS_DETECTOR_REFERENCE_AREA_PDF
 * (the reference's doubled term). */
WOS_API int wos_boundary_term(wos_scene_t scene, const wos_detector *det, int nwalks, uint64_t seed,
                              const float *dV_dir, double *image_tangent, const float *dLdI, float *dV,
                              wos_stream_t stream);

/* ---------------------------------------------------------------- batched */

/* One (scene, query set) of a batch.  P (n x dim) and target_or_dLdu stay at
 * their device addresses for the batch's lifetime (a captured graph reads
 * them in place); their contents may change between runs.  loss_kind as in
 * wos_solve_adjoint. */
typedef struct wos_batch_item {
    wos_scene_t scene;
    const float *P;
    int32_t n;
    int32_t loss_kind;
    const float *target_or_dLdu;
    wos_params params;
} wos_batch_item;

typedef struct wos_batch_s *wos_batch_t;

/* Plan a batched forward (+ adjoint if want_adjoint) over many items: items
 * of one dimension form a group whose walks are concatenated in order of the
 * scenes' tree depth, then item order (order the items scene-major); each
 * walk phase runs one persistent work-queue launch per run of equal depth
 * (compiled for that depth), the reductions one launch per group.
 * wos_batch_info reports the number of groups (dimensions present).
 * Buffers for all outputs are owned by the plan (wos_batch_outputs).  The
 * plan reads the items' scenes, points and targets in place at every run:
 * they must outlive it (destroy the plan before its scenes).  This
 * is the batched form of wos_solve_adjoint; no counterpart in the reference,
 * whose callers loop over scenes with one thrust launch each
 * (include/wos.cuh:407-440). */
WOS_API int wos_batch_create(const wos_batch_item *items, int n_items, const wos_adjoint_params *a, int want_adjoint,
                             wos_stream_t stream, wos_batch_t *out);

/* Launch shape of the batch kernels (see wos_launch_config). */
WOS_API int wos_batch_set_launch(wos_batch_t b, int block_threads, int blocks_per_sm, int chunk);

/* Launch-shape autotuner: times whole steps of the plan (no graph) for each
 * candidate (block_threads[i], chunk[i]) on `stream` with CUDA events -- one
 * untimed step, then the best of `repeats` -- and keeps the fastest with
 * wos_batch_set_launch (blocks per SM unchanged).  Results do not depend on
 * the shape, only speed does.  ms (n_candidates floats, may be NULL) gets each
 * candidate's time, *best its index.  Synchronises the stream, so it must not
 * be called while the stream is being captured.  This library's own tuner;
 * no counterpart in the reference, whose launch shape is fixed. */
WOS_API int wos_batch_autotune(wos_batch_t b, const int32_t *block_threads, const int32_t *chunk, int n_candidates,
                               int repeats, wos_stream_t stream, float *ms, int32_t *best);

/* Slot-wise launch-shape tuner: the plan keeps one launch shape per slot
 * (dimension 2 or 3 x phase: walks, adjoint); after one full step it times,
 * for each slot present, that slot's launches alone over the first `sample`
 * fraction (0 < sample <= 1) of every run's walks for each candidate
 * (block_threads[i], blocks_per_sm[i] (0 = occupancy limit), chunk[i]) --
 * the best of `repeats` -- and keeps the fastest for that slot.  ms
 * (4 x n_candidates floats, slot k = (dim - 2) * 2 + phase; NaN for absent
 * slots) and best (4 indices, -1 for absent slots) may be NULL.  Results do
 * not depend on the shapes.  Synchronises the stream; not during capture.
 * No counterpart in the reference. */
WOS_API int wos_batch_autotune_slots(wos_batch_t b, const int32_t *block_threads, const int32_t *blocks_per_sm,
                                     const int32_t *chunk, int n_candidates, int repeats, double sample,
                                     wos_stream_t stream, float *ms, int32_t *best);

/* Set the launch shape of one slot (dim 2 or 3, phase 0 walks / 1 adjoint). */
WOS_API int wos_batch_set_launch_slot(wos_batch_t b, int dim, int phase, int block_threads, int blocks_per_sm,
                                      int chunk);

/* The launch shape of slot (dim, phase 0 walks / 1 adjoint): out[0] threads
 * per block, out[1] blocks per SM (0 = occupancy limit), out[2] chunk. */
WOS_API int wos_batch_get_launch(wos_batch_t b, int dim, int phase, int32_t *out);

/* Re-read the scenes' device views.  wos_batch_run does this by itself for
 * scenes rebuilt (wos_scene_update_vertices) or given a new source
 * (wos_scene_set_source) since the last read, and then captures its graph
 * anew; this call forces it. */
WOS_API int wos_batch_refresh(wos_batch_t b, wos_stream_t stream);

/* Run one step.  use_graph != 0: the step is captured once into a CUDA graph
 * (on the first call) and replayed with one graph launch per call. */
WOS_API int wos_batch_run(wos_batch_t b, int use_graph, wos_stream_t stream);

/* Device pointers to item `item`'s outputs: per-point mean / var (double),
 * its loss (double), gradients dV (nV x dim), dg (nV), dsrc (5) (float, NULL
 * without adjoint).  Valid until wos_batch_destroy. */
WOS_API int wos_batch_outputs(wos_batch_t b, int item, const double **mean, const double **var, const double **loss,
                              const float **dV, const float **dg, const float **dsrc);

/* Copy item `item`'s outputs into caller buffers (device; any may be NULL). */
WOS_API int wos_batch_copy_outputs(wos_batch_t b, int item, double *mean, double *var, double *loss, float *dV,
                                   float *dg, float *dsrc, wos_stream_t stream);

WOS_API int wos_batch_info(wos_batch_t b, int64_t *total_walks, int64_t *total_points, int32_t *n_groups);
WOS_API int wos_batch_destroy(wos_batch_t b, wos_stream_t stream);

/* ---------------------------------------------------------------- no allocation */

/* Largest n * nwalks that wos_solve_noalloc accepts. */
#define WOS_NOALLOC_MAX_WALKS 4194304

/* wos_solve without any device allocation, for callers that may not
 * allocate device memory (applications that own the device through their
 * own pool and forbid plug-ins from calling cudaMalloc, latency-critical
 * loops that cannot take its implicit synchronisation, processes under a
 * hard device-memory quota).  No counterpart in the reference.
 *
 * Scratch is a fixed array inside the library: 16 MiB + 256 bytes on every
 * GPU that loads it, held until the process exits.  n * nwalks must not
 * exceed WOS_NOALLOC_MAX_WALKS; larger requests fail with WOS_ERR_WORKSPACE
 * and a message (split the points, or use wos_solve).  Every call looks up
 * the array's device address with the caller's device current (so a device
 * reset between calls is harmless); the first call on a device may also load
 * the library's device code there, so make that first call before any stream
 * capture.  All calls share the one
 * array, so calls that overlap on the GPU (concurrent streams or threads)
 * race on it: order them on one stream.  Results equal wos_solve's. */
WOS_API int wos_solve_noalloc(wos_scene_t scene, const float *P, int n, const wos_params *p, double *mean, double *var,
                              wos_stream_t stream);

/* ---------------------------------------------------------------- kernels */

/* Launch shape of the persistent walk kernels: threads per block, blocks per
 * SM (0 = occupancy limit), walks taken per queue grab, LBVH nodes staged in
 * shared memory per block.  In wos_set_launch_config, block_threads = 0,
 * chunk = 0, blocks_per_sm < 0 and smem_nodes < 0 keep the current value. */
typedef struct wos_launch_config {
    int32_t block_threads;
    int32_t blocks_per_sm;
    int32_t chunk;
    int32_t smem_nodes;
} wos_launch_config;

/* Work accounting: while enabled, the persistent walk and adjoint kernels add
 * their nearest-query totals to a device counter {queries, LBVH node visits,
 * primitive distance evaluations} (brute force: nF evaluations per query).
 * wos_work_counters reads it (synchronising the device); reset != 0 clears.
 * While enabled those kernels run an instance compiled with counters (one for
 * every tree depth); the default instances carry none, which saves 1-3 % of a
 * step.  Results are the same either way. */
WOS_API int wos_set_work_counting(int enable);
WOS_API int wos_work_counters(int reset, int64_t *out);

/* Order in which the adjoint kernel runs the samples of wos_solve_adjoint and
 * wos_solve_tangent.  mode 1 (default): sorted by the position of each walk's
 * boundary primitive in the scene's primitive order (one radix sort of the
 * walk records per call), so samples that start next to each other run
 * together and share the tree's cached leaves; mode 0: in (point, walk)
 * order.  Results are the same in both modes up to the summation order of
 * the FP64 gradient sums.  The mode changes the workspace size: query the
 * *_workspace_size functions after setting it.  No counterpart in the
 * reference (one thread per walk, in launch order). */
WOS_API int wos_set_sample_order(int mode);

WOS_API int wos_set_launch_config(int dim, const wos_launch_config *cfg);
WOS_API int wos_get_launch_config(int dim, wos_launch_config *out);

/* Reference-style walk kernel: one thread per (point, walk), no walk
 * regeneration, no shared-memory staging -- the shape of the reference's
 * thrust::for_each launch (include/wos.cuh:407-440).  Same values as
 * wos_walk_values; kept as the comparison kernel. */
WOS_API int wos_walk_values_plain(wos_scene_t scene, const float *P, int n, const wos_params *p, float *values,
                          wos_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* WOS_B200_H */
