/*
 * catsurf_b200.h -- C ABI of the B200-native CAT-Surface hot paths.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream, returns an
 * int status (CSG_OK == 0, negative CSG_ERR_* otherwise) and never throws.
 * Device pointers are owned by the caller; kernels that need working memory
 * take a caller-provided `scratch` buffer whose size is given by the matching
 * *_scratch_bytes() query.  csg_last_error() returns a thread-local message
 * for the last failure on the calling thread.
 *
 * Each declaration names the reference interface it replaces
 * (paths relative to the reference project root).
 */
#ifndef CATSURF_B200_H
#define CATSURF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CSG_API __attribute__((visibility("default")))
#else
#define CSG_API
#endif

/* Binary-compatible with cudaStream_t; 0 selects the legacy default stream. */
typedef struct CUstream_st *csg_stream_t;

#define CSG_OK 0
#define CSG_ERR_ARG (-1)         /* invalid argument or shape */
#define CSG_ERR_CUDA (-2)        /* CUDA runtime error */
#define CSG_ERR_TIMEOUT (-3)     /* a bounded device-side wait ran out */
#define CSG_ERR_LAUNCH (-4)      /* the grid cannot be made co-resident */
#define CSG_ERR_TOPOLOGY (-5)    /* face indices out of range / not a mesh */
#define CSG_ERR_UNSUPPORTED (-6) /* option not supported */
#define CSG_ERR_COVERAGE (-7)    /* a query point found no candidate triangle */
#define CSG_ERR_FORMAT (-8)      /* a file payload that does not decode */

#define CSG_DTYPE_F32 0 /* DARTEL / warp element type */
#define CSG_DTYPE_F64 1

#define CSG_ARITH_CAT 0  /* float32 storage, CAT mixed float32/float64 arithmetic */
#define CSG_ARITH_FP32 1 /* float32 storage and arithmetic */
#define CSG_ARITH_FP64 2 /* float64 storage and arithmetic */

CSG_API const char *csg_last_error(void);
CSG_API int csg_abi_version(void);
/* Kernels this library has launched in this process (every entry point
 * counts its own launches; launches replayed from a captured CUDA graph are
 * not seen here). */
CSG_API long long csg_kernel_launches(void);

/* ------------------------------------------------------------------------
 * Surf2Sphere: mesh topology (host, no device memory).
 * ---------------------------------------------------------------------- */

/* Incident-face CSR, faces in ascending id per vertex.
 * Replaces Surf2SphereTopology.from_mesh incidence
 * (src/cat_surface_gpu/surf2sphere.py:412-436).
 * inc_off: [n_vertices + 1]; inc_face: [3 * n_faces]. */
CSG_API int csg_mesh_incidence(int n_vertices, const int32_t *faces, int n_faces, int32_t *inc_off, int32_t *inc_face);

/* Unique, ascending 1-ring neighbour CSR.
 * Replaces _build_neighbour_table (src/cat_surface_gpu/surface_stencil.py:36-66).
 * nbr_off: [n_vertices + 1]; nbr: capacity >= 6 * n_faces.
 * Returns the number of directed edges written (>= 0) or an error. */
CSG_API int csg_mesh_neighbours(int n_vertices, const int32_t *faces, int n_faces, int32_t *nbr_off, int32_t *nbr,
                        int nbr_capacity);

/* Greedy first-fit colouring in vertex order over a neighbour CSR: vertex v
 * takes the smallest colour none of its already coloured neighbours has.
 * Replaces _build_color_groups (src/cat_surface_gpu/surface_stencil.py:69-91).
 * colour_off [n_vertices + 1] (first n_colours + 1 used), members
 * [n_vertices] (each colour's vertices ascending).  Returns n_colours or a
 * negative CSG_ERR_*. */
CSG_API int csg_colour_groups(int n_vertices, const int32_t *nbr_off, const int32_t *nbr, int32_t *colour_off,
                              int32_t *members);

/* Centre a sphere on its vertex mean (the sequential float64 sum of the
 * float32 coordinates over n) and project every vertex to unit length, in
 * float64 with a float32 result (host; replaces _normalise_sphere,
 * src/cat_surface_gpu/gpu_pipeline.py:274-305).  A vertex of zero or
 * non-finite length is CSG_ERR_ARG. */
CSG_API int csg_normalise_sphere(int n_vertices, const float *in, float *out);

/* level(v) = 1 + max level of lower-index neighbours (0 if none).
 * Replaces _build_ordered_dependency_groups
 * (src/cat_surface_gpu/surface_stencil.py:94-109).  Returns the level count. */
CSG_API int csg_dependency_levels(int n_vertices, const int32_t *nbr_off, const int32_t *nbr, int32_t *levels);

/* Greedy colouring in vertex order.  Replaces _build_color_groups
 * (src/cat_surface_gpu/surface_stencil.py:69-91).  Returns the colour count. */
CSG_API int csg_greedy_colours(int n_vertices, const int32_t *nbr_off, const int32_t *nbr, int32_t *colours);

/* Wavefront plan for the ordered sweeps (host).
 * Vertex v of sweep s runs at wavefront step s * level_stride + level(v),
 * where level() is any integer schedule with 1 <= level(w) - level(v) <=
 * level_stride - 1 on every edge v < w; that keeps exactly the sequential
 * Gauss-Seidel reads (lower neighbours of the current sweep, higher
 * neighbours of the previous one).  The builder starts from the longest-path
 * levels and lowers the stride while difference-constraint relaxation still
 * finds a schedule (61,442-vertex hull: stride 11 -> 6, so 45% fewer steps).
 * Outputs: slot_off [n+1]; slot_tri [3 * n_faces * 4] (per incident slot the
 * face's three vertex ids in face order plus the face id, int4-aligned);
 * order [n] (vertices sorted by (level mod stride, level, id));
 * level_begin / level_end [n] (range of each level inside `order`). */
typedef struct {
    int32_t n_vertices;
    int32_t n_faces;
    int32_t n_levels;
    int32_t level_stride;
    int32_t max_degree;
    int32_t n_slots;
} csg_areal_plan_info;

CSG_API int csg_areal_plan_build(int n_vertices, const int32_t *faces, int n_faces, int32_t *slot_off, int32_t *slot_tri,
                         int32_t *order, int32_t *level_begin, int32_t *level_end, csg_areal_plan_info *info);

/* ------------------------------------------------------------------------
 * Surf2Sphere: the 4,999 ordered area-smoothing sweeps (device).
 * Replaces run_areal_smoothing_cuda's sweep loop and the Triton kernels
 * _areal_smoothing_kernel / _normalize_points_kernel
 * (src/cat_surface_gpu/surf2sphere.py:35-280, 940-1104): sweeps
 * 1 .. iterations-1, projection to `radius` after sweep s when
 * s % project_every == 0.  One persistent cooperative launch.
 * points: device float32 [n,3] (CSG_ARITH_CAT / _FP32) or float64 [n,3]
 * (CSG_ARITH_FP64), updated in place.  Plan arrays are device copies of
 * csg_areal_plan_build's outputs (max_degree from its info: the largest
 * incident-face count; each CTA caches its vertices' face slots in shared
 * memory when they fit).  n_ctas / threads_per_cta /
 * lanes_per_vertex of 0 pick defaults; timeout_s bounds every device wait.
 * The kernel's status lands in scratch; read it with csg_read_status.
 * ---------------------------------------------------------------------- */
/* Scratch bytes for csg_areal_sweeps; 0 for n_vertices < 1 or an unknown arithmetic. */
CSG_API size_t csg_areal_scratch_bytes(int n_vertices, int arithmetic);

CSG_API int csg_areal_sweeps(void *points, int n_vertices, const int32_t *slot_off, const int32_t *slot_tri,
                     const int32_t *order, const int32_t *level_begin, const int32_t *level_end, int n_levels,
                     int level_stride, int max_degree, int iterations, int project_every, double radius, int arithmetic, void *scratch,
                     size_t scratch_bytes, int n_ctas, int threads_per_cta, int lanes_per_vertex, double timeout_s,
                     csg_stream_t stream);

/* Allocation-free variant of csg_areal_sweeps (no counterpart in the
 * reference).  Some callers cannot call cudaMalloc: code running while a CUDA
 * stream capture is active on its thread, hosts that give all device memory
 * to their own pool allocator up front, and foreign-function bindings that
 * own no device allocator.  This entry point takes the same inputs and
 * in/out points as csg_areal_sweeps but no scratch: its working memory is a
 * file-scope device array of 4 MiB + 256 bytes that every GPU loading the
 * library holds until exit, so it handles at most 262,144 vertices in the
 * float32 modes and 131,072 in CSG_ARITH_FP64 (larger meshes are rejected
 * with CSG_ERR_ARG before any device work).  It allocates nothing.  The first
 * call on each device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the one array, so calls that overlap on the GPU (other
 * streams, other threads) race; serialise them.  With status_out non-NULL the
 * call waits for the kernel and reports its status word (also returned);
 * with NULL it returns once the work is enqueued.  status_out must be NULL
 * while `stream` is being captured (CSG_ERR_ARG otherwise, before any work).
 * The array's address is looked up once per device, so the library must not
 * be used across a cudaDeviceReset of that device. */
CSG_API int csg_areal_sweeps_noalloc(void *points, int n_vertices, const int32_t *slot_off, const int32_t *slot_tri,
                                     const int32_t *order, const int32_t *level_begin, const int32_t *level_end,
                                     int n_levels, int level_stride, int max_degree, int iterations, int project_every,
                                     double radius, int arithmetic, int n_ctas, int threads_per_cta,
                                     int lanes_per_vertex, double timeout_s, int *status_out, csg_stream_t stream);

/* Self-test of the bounded device-side wait (no reference counterpart): a
 * 2-CTA cooperative grid waits on a barrier that expects one arrival more
 * than the grid has; the wait gives up after timeout_s (<= 10 s) and records
 * CSG_ERR_TIMEOUT in scratch's status word.  Exercises the timeout path
 * without faulting or hanging the GPU; the context stays usable. */
/* Self-test of the kernels' division by three (two multiplies, see
 * csrc/common.cuh): writes __ddiv_rn(x, 3) and the fast form for n values so
 * a test can compare them bit for bit.  No reference counterpart. */
CSG_API int csg_selftest_div3(const double *x, long long n, double *by_division, double *by_multiplies,
                              csg_stream_t stream);

CSG_API int csg_selftest_barrier_timeout(void *scratch, size_t scratch_bytes, double timeout_s, csg_stream_t stream);

/* Surf2Sphere stages 1-5 (low_smooth, inflate, very_inflate, high_smooth,
 * ellipsoid) in place on float32 points [n][3] (device), stages 1..stop_at.
 * Replaces run_surf2sphere_preprocess_cuda
 * (src/cat_surface_gpu/surf2sphere.py:716-862) without the final
 * ellipsoid-to-sphere conversion (host).  Distance-smoothing passes run in
 * vertex-index Gauss-Seidel order (the upstream binary's) as persistent
 * wavefront launches over the sweep schedule (order, level ranges, stride of
 * csg_areal_plan_build); nb_off/nb: unique ascending 1-ring; inc_off/inc:
 * per-vertex incidences face << 2 | corner sorted by (corner, face).
 * Float32 storage, float64 arithmetic.  The inflation is a pointwise pass of
 * the same wavefront, so a launch ends only at a global step (stage
 * statistics, distortion selection): 19 launches for stages 1-5.
 * max_degree: the largest 1-ring (nb_off[v+1] - nb_off[v]); > 0 lets each
 * CTA keep its vertices' rings in shared memory, 0 reads them from global
 * memory.  A ring longer than max_degree sets status CSG_ERR_ARG.  Waits are
 * bounded by timeout_s (status CSG_ERR_TIMEOUT in the scratch's control
 * block, read with csg_read_status). */
/* convert_ellipsoid_to_sphere_with_surface_area (src/cat_surface_gpu/
 * surf2sphere.py:919-937) in place on device float32 points [n][3]:
 * half-axes a = (|min| + |max|) / 2 per coordinate (float32, at least 1e-20),
 * then x <- radius x / |x / a| / a in float64 (radius = sqrt(area / (4 pi))),
 * stored as float32; equal to the reference's NumPy arithmetic.  scratch:
 * 16 bytes of device memory. */
CSG_API int csg_ellipsoid_to_sphere(float *points, int n, double radius, void *scratch, size_t scratch_bytes,
                                    csg_stream_t stream);
CSG_API size_t csg_preprocess_scratch_bytes(int n_vertices, int n_faces);
CSG_API int csg_surf2sphere_preprocess(float *points, int n, const int32_t *faces, int n_faces,
                                       const int32_t *nb_off, const int32_t *nb, const int32_t *inc_off,
                                       const int32_t *inc, const int32_t *order, const int32_t *level_begin,
                                       const int32_t *level_end, int n_levels, int level_stride, int max_degree,
                                       int stop_at, void *scratch, size_t scratch_bytes, int n_ctas,
                                       int threads_per_cta, int lanes_per_vertex, double timeout_s,
                                       csg_stream_t stream);

/* ------------------------------------------------------------------------
 * SurfWarp rotation feature: the depth potential (device, batched).
 * Replaces compute_rotation_feature's solve (src/cat_surface_gpu/
 * rotation_feature.py:37-317): stable normals, mixed Voronoi areas, the
 * cotangent system (L + alpha A) u = (H - mean H) A with H the mean
 * curvature, solved by coloured SOR (relaxation, max_iter sweeps) or
 * Jacobi-preconditioned CG (max_iter, tolerance on |r| / |rhs|).
 * geometry: device float32 [batch][n][3] (the smoothed coarse surfaces of one
 * triangulation); faces [nf][3]; inc_off/inc: per-vertex incidences
 * face << 2 | corner sorted by (corner, face) (csg_mesh_incidence order);
 * max_incidences: the largest incidence count.  Rows sum in the order of the
 * reference's CPU index_add_, so each row, normal, area and SOR sweep equals
 * the reference's float64 CPU result; whole-vector sums are blocked (runs of
 * 256, 32 lanes, pairwise) and do not depend on the launch shape.
 * SOR needs the wavefront schedule of the colour-major order: relabel the
 * vertices by (colour of csg_colour_groups, id), build csg_areal_plan_build's
 * schedule on the relabelled faces, map its order back to the original ids.
 * Outputs (device): values [batch][n] (the raw potential, before the
 * reference's smoothing and min-max normalisation), iterations [batch],
 * residual [batch] (|rhs - A u| / |rhs|); normals [batch][n][3] and areas
 * [batch][n] when non-NULL.  alpha must be non-zero.  Waits are bounded by
 * timeout_s (status in the scratch's control block, csg_read_status).
 * ---------------------------------------------------------------------- */
#define CSG_DEPTH_SOR 0
#define CSG_DEPTH_PCG 1
CSG_API size_t csg_depth_scratch_bytes(int n_vertices, int n_faces, int batch);
CSG_API int csg_depth_potential(const float *geometry, int batch, int n, const int32_t *faces, int nf,
                                const int32_t *inc_off, const int32_t *inc, int max_incidences, double alpha,
                                int solver, int max_iter, double tolerance, double relaxation, const int32_t *order,
                                const int32_t *level_begin, const int32_t *level_end, int n_levels,
                                int level_stride, double *values, int32_t *iterations, double *residual,
                                double *normals, double *areas, void *scratch, size_t scratch_bytes, int n_ctas,
                                int threads_per_cta, int lanes_per_row, double timeout_s, csg_stream_t stream);

/* ------------------------------------------------------------------------
 * SurfWarp: 2-D DARTEL on the lat-lon sheet (device, batched).
 * Fields are [batch][channels][ny][nx] of dtype CSG_DTYPE_F32 / _F64; maps
 * are one-based coordinates [2], Jacobians (j00, j10, j01, j11) [4],
 * gradients [2], Hessians (h00, h11, h01) [3].  Arithmetic follows the
 * reference's torch path operation by operation (one rounding each).
 * params are the five regulariser values (sx, sy, mu, lambda, identity).
 * ---------------------------------------------------------------------- */

/* Data term E_b(v) = 1/2 sum_x (S_b(exp(v_b)(x)) - T_b(x))^2, exp(v) by k
 * scaling-and-squaring compositions (expdef's maps), and its exact adjoint
 * (no reference counterpart: a hand-written adjoint of DARTEL's data term;
 * the reference's Gauss-Newton gradient of the same term is
 * initialise_objfun + squaring_update, dartel_grid.py:723-914).
 * Checkpoints: the forward keeps phi_0, phi_c, phi_2c, ... (c =
 * checkpoint_every; csg_dartel_data_checkpoints maps of [batch][2][ny][nx]);
 * the backward recomputes the maps between checkpoints.  objective [batch];
 * grad_velocity [batch][2][ny][nx] = grad_scale[b] dE_b/dv_b (grad_scale a
 * device array [batch] or NULL for 1).  The value scatter of each
 * composition step uses atomic adds, so gradients agree across runs to
 * rounding, not bit for bit. */
CSG_API size_t csg_dartel_data_scratch_bytes(int dtype, int batch, int nx, int ny, int k, int checkpoint_every);
CSG_API int csg_dartel_data_checkpoints(int k, int checkpoint_every);
CSG_API int csg_dartel_data_forward(int dtype, int batch, int nx, int ny, const void *velocity, const void *source,
                                    const void *target, int k, int checkpoint_every, void *checkpoints,
                                    void *objective, void *scratch, size_t scratch_bytes, csg_stream_t stream);
CSG_API int csg_dartel_data_backward(int dtype, int batch, int nx, int ny, const void *source, const void *target,
                                     int k, int checkpoint_every, const void *checkpoints, const void *grad_scale,
                                     void *grad_velocity, void *scratch, size_t scratch_bytes, csg_stream_t stream);

/* Scratch for csg_dartel_solve / _step / _fmg / _expdef / _squaring / _objfun. */
CSG_API size_t csg_dartel_scratch_bytes(int dtype, int batch, int nx, int ny);

/* Whole solve of `batch` independent (source, target) sheet pairs:
 * for index in 0..loop-1, its times dartel_step(k = index, params[index]).
 * velocity [batch][2][ny][nx] in/out (zeros for the reference's start);
 * metrics [batch][loop*its][3] (objective, regulariser/2, |rhs|).
 * Replaces the eager loop of solve_dartel_maps
 * (src/cat_surface_gpu/surface_warp.py:321-353) and dartel_step
 * (src/cat_surface_gpu/dartel_grid.py:1420-1616).  With
 * assume_initial_nonzero the call makes no host synchronisation and can be
 * captured in a CUDA graph. */
CSG_API int csg_dartel_solve(int dtype, int batch, int nx, int ny, const void *source_maps, const void *target_maps,
                             void *velocity, void *metrics, int loop, const double *params, int its, double lmreg,
                             int cycles, int nit, int code, int assume_initial_nonzero, void *scratch,
                             size_t scratch_bytes, csg_stream_t stream);

/* One dartel_step (dartel_grid.py:1420-1616), rtype 1, no distortion. */
CSG_API int csg_dartel_step(int dtype, int batch, int nx, int ny, const void *source, const void *target,
                            void *velocity, void *metrics, int k, const double *params, double lmreg, int cycles,
                            int nit, int code, int assume_initial_nonzero, void *scratch, size_t scratch_bytes,
                            csg_stream_t stream);

/* smalldef_jac / jacobian_of_displacement (dartel_grid.py:624-675):
 * map = id + v * scale, jac = I + central differences of v * scale / 2.
 * Either output may be NULL. */
CSG_API int csg_dartel_smalldef(int dtype, int batch, int nx, int ny, const void *velocity, double scale,
                                void *map_out, void *jac_out, csg_stream_t stream);

/* composition / composition_jacobian (dartel_grid.py:407-507, 534-587):
 * c = b o a with period unwrapping; jc = J_b(a) J_a.  ja, jb, jc_out are all
 * NULL (map only) or all set. */
CSG_API int csg_dartel_compose(int dtype, int batch, int nx, int ny, const void *a, const void *ja, const void *b,
                               const void *jb, void *c_out, void *jc_out, csg_stream_t stream);

/* jac_div_smalldef (dartel_grid.py:678-720). */
CSG_API int csg_dartel_jac_div(int dtype, int batch, int nx, int ny, const void *jac, const void *velocity,
                               double scale, void *out, csg_stream_t stream);

/* initialise_objfun (dartel_grid.py:723-775); weights may be NULL;
 * objective_out [batch]. */
CSG_API int csg_dartel_objfun(int dtype, int batch, int nx, int ny, const void *source, const void *target,
                              const void *map, const void *jac, const void *weights, void *rhs_out, void *hess_out,
                              void *objective_out, void *scratch, size_t scratch_bytes, csg_stream_t stream);

/* squaring_update (dartel_grid.py:778-914; dartel_triton.py:345-477) with
 * the reference's scratch slot (return_scratch); map/jac/scratch outputs may
 * be NULL. */
CSG_API int csg_dartel_squaring(int dtype, int batch, int nx, int ny, const void *rhs, const void *hess,
                                const void *map, const void *jac, int k, int save_transformation, void *b_out,
                                void *a_out, void *map_out, void *jac_out, void *scratch_map_out, void *scratch,
                                size_t scratch_bytes, csg_stream_t stream);

/* regularization_operator rtype 0 / 1 / 2 (dartel_grid.py:917-1015). */
CSG_API int csg_dartel_regularization(int dtype, int batch, int nx, int ny, const void *velocity,
                                      const double *params, int rtype, void *out, csg_stream_t stream);

/* apply_membrane_system (dartel_grid.py:1018-1070; dartel_triton.py:190-239). */
CSG_API int csg_dartel_membrane_apply(int dtype, int batch, int nx, int ny, const void *hess, const void *field,
                                      const double *params, void *out, csg_stream_t stream);

/* relax_membrane: nit red-black sweeps in place (dartel_grid.py:1073-1208;
 * dartel_triton.py:242-291, 606-640).  Needs an even nx (or nx == 1), as the
 * reference's CUDA path does. */
CSG_API int csg_dartel_relax(int dtype, int batch, int nx, int ny, const void *hess, const void *rhs,
                             const double *params, int nit, void *u, csg_stream_t stream);

/* resize_field: separable quadratic B-spline (dartel_grid.py:239-305;
 * dartel_triton.py:59-187); `fields` = batch * channels; accumulate adds. */
CSG_API int csg_dartel_resize(int dtype, int fields, int src_nx, int src_ny, const void *src, int dst_nx, int dst_ny,
                              void *dst, int accumulate, csg_stream_t stream);

/* fmg2_membrane (dartel_grid.py:1211-1417); u holds the initial guess when
 * has_initial, else it is overwritten. */
CSG_API int csg_dartel_fmg(int dtype, int batch, int nx, int ny, const void *hess, const void *rhs,
                           const double *params, int cycles, int nit, void *u, int has_initial,
                           int assume_initial_nonzero, void *scratch, size_t scratch_bytes, csg_stream_t stream);

/* expdef: scaling and squaring of id + v / 2^k (dartel_grid.py:1619-1666);
 * jac_out may be NULL. */
CSG_API int csg_dartel_expdef(int dtype, int batch, int nx, int ny, const void *velocity, int k, void *map_out,
                              void *jac_out, void *scratch, size_t scratch_bytes, csg_stream_t stream);

/* sample_field: bilinear samples of a [ny][nx] field at n (x, y) points,
 * zero-based, with the DARTEL boundary rule (dartel_grid.py:590-621). */
CSG_API int csg_dartel_sample(int dtype, int nx, int ny, const void *field, int n, const void *x, const void *y,
                              void *out, csg_stream_t stream);

/* apply_flow_to_sphere with unit-sphere points (float32 [n][3]) and a flow
 * [2][ny][nx]; out [n][3] of the flow's dtype (surface_warp.py:500-617). */
CSG_API int csg_apply_flow_to_sphere(int dtype, int n, const float *unit_points, int nx, int ny, const void *flow,
                                     int inverse, void *out, csg_stream_t stream);

/* -avg blend of the x- and z-pole warped spheres, float64 [n][3] in, float32
 * [n][3] out (src/cat_surface_gpu/gpu_pipeline.py:248-271). */
CSG_API int csg_average_xz(int n, const double *x_surface, const double *z_surface, float *out, csg_stream_t stream);

/* ------------------------------------------------------------------------
 * SurfWarp: initial-rotation search (host grid index, device costs).
 * ---------------------------------------------------------------------- */

/* Uniform grid over [-1, 1]^3 of grid_size^3 cells; each triangle is listed,
 * in face order, in every cell its bounding box (+/- margin cells) covers.
 * Replaces RotationGridIndex.from_geometry
 * (src/cat_surface_gpu/surface_rotation.py:58-120).  offsets
 * [grid_size^3 + 1]; with cell_faces NULL only offsets and *count are
 * produced (size query). */
CSG_API int csg_rotation_grid_build(const double *points, int n_points, const int32_t *faces, int n_faces,
                                    int grid_size, int margin, int32_t *offsets, int32_t *cell_faces,
                                    long long capacity, long long *count);

/* The same grid built on the device (device points, faces, offsets and
 * cell_faces; scratch of csg_rotation_grid_scratch_bytes()): counts, scan,
 * fill and a per-cell sort, so every cell lists its faces in ascending order
 * exactly as csg_rotation_grid_build does.  *count is read back (the call
 * synchronises `stream`); with cell_faces NULL only offsets and *count are
 * produced. */
CSG_API size_t csg_rotation_grid_scratch_bytes(int grid_size);
CSG_API int csg_rotation_grid_build_device(const double *points, int n_points, const int32_t *faces, int n_faces,
                                           int grid_size, int margin, int32_t *offsets, int32_t *cell_faces,
                                           long long capacity, long long *count, void *scratch, size_t scratch_bytes,
                                           csg_stream_t stream);

/* One surface of a batched cost evaluation (all device pointers).  With
 * n_features F > 1 the cost sums the squared differences of all F features
 * (feature-major: src_values [F][n_src], tgt_values [F][n_tgt_points]);
 * n_features 0 or 1 is the reference's single feature. */
typedef struct {
    const float *src_points;     /* [n_src][3] source sphere points */
    const double *src_values;    /* [n_features][n_src] source features */
    const float *triangles;      /* [n_tri][9] target triangle corners */
    const int32_t *faces;        /* [n_tri][3] target faces */
    const double *tgt_values;    /* [n_features][n_tgt_points] target features */
    const int32_t *grid_offsets; /* csg_rotation_grid_build offsets */
    const int32_t *grid_faces;   /* csg_rotation_grid_build cell faces */
    const float *matrices;       /* [n_candidates][9] column-major rotations */
    int32_t n_src;
    int32_t grid_size;
    int32_t n_candidates;
    int32_t n_features;          /* 0 or 1: one feature */
    int32_t n_tgt_points;        /* feature stride of tgt_values (needed when n_features > 1) */
    const float *records;        /* optional [n_tri][20] csg_rotation_triangle_records of `triangles`
                                    (16-byte aligned); NULL: the same terms are formed per query and
                                    every candidate of the cell is tested */
} csg_rotation_surface;

/* Per-triangle terms of the closest-polygon test, once per target sphere
 * (ABI version 3): record t = corners p0, p1, p2 (9 floats), n = (p1 - p0) x
 * (p2 - p0) (3), n.n, |p1 - p0|^2, (p1 - p0).(p2 - p0), |p2 - p0|^2 -- the
 * float32 values the cost kernel would otherwise form for every query and
 * triangle, with the same operations -- then a bounding sphere (centre 3,
 * radius 1) that covers every point the tolerant test can return.  With
 * records the kernel tests first the candidate nearest by its sphere and skips
 * every candidate whose sphere lies clearly farther than that distance: none
 * of those can be the first minimum, so the costs are identical either way.
 * triangles: device [n_tri][9]; records: device [n_tri][20], 16-byte
 * aligned.  No reference counterpart (the reference tests every candidate). */
CSG_API int csg_rotation_triangle_records(const float *triangles, int n_tri, float *records, csg_stream_t stream);

CSG_API size_t csg_rotation_scratch_bytes(int n_surfaces, const int *n_src, const int *n_candidates, int tile);

/* SSD cost of every candidate rotation of every surface in one persistent
 * launch: closest target triangle of each rotated source point (plane
 * projection with a 1e-3 inside tolerance, else nearest edge), barycentric
 * resampling of the target feature, float64 sum of squared differences.
 * costs: concatenated [n_candidates] per surface.  tile (128/256/512) is the
 * number of source points per work item; n_ctas 0 = fill the GPU.
 * Replaces RotationGridIndexDevice.cost_batch_prepared
 * (src/cat_surface_gpu/surface_rotation.py:354-546).  A query point whose
 * cell has no candidate triangle sets CSG_ERR_COVERAGE (read with
 * csg_rotation_status). */
CSG_API int csg_rotation_cost_batch(int n_surfaces, const csg_rotation_surface *surfaces, double *costs, int tile,
                                    int n_ctas, void *scratch, size_t scratch_bytes, csg_stream_t stream);

/* Byte offset in the scratch of csg_rotation_cost_batch(n_surfaces, ...) of the
 * int coverage status that csg_rotation_status reads (0 for n_surfaces < 1), so
 * a caller can copy it with its own asynchronous readback.  No reference
 * counterpart. */
CSG_API size_t csg_rotation_status_offset(int n_surfaces);

/* Synchronously read the coverage status of the last csg_rotation_cost_batch
 * that used this scratch (CSG_OK or CSG_ERR_COVERAGE). */
CSG_API int csg_rotation_status(const void *scratch, int n_surfaces, csg_stream_t stream, int *status);

/* One surface's costs for a few candidates whose matrices are in host memory,
 * for searches that decide on the host between evaluations (the reference's
 * Nelder-Mead loop calls cost_batch_prepared once per decision,
 * src/cat_surface_gpu/surface_rotation.py:650-699).  Copies the
 * surface->n_candidates (1 .. CSG_ROTATION_HOST_MAX_CANDIDATES) float32
 * matrices from `matrices_host` (page-locked for an asynchronous copy) to
 * `matrices_device`, which replaces surface->matrices, runs
 * csg_rotation_cost_batch (one surface; scratch sized by
 * csg_rotation_scratch_bytes), copies the coverage status (int32 at byte 0)
 * and the float64 costs (from byte 8) to `readback_host`
 * (8 + 8 * n_candidates bytes) and synchronises `stream`. */
#define CSG_ROTATION_HOST_MAX_CANDIDATES 31
CSG_API int csg_rotation_cost_host(const csg_rotation_surface *surface, const float *matrices_host,
                                   float *matrices_device, void *readback_host, int tile, void *scratch,
                                   size_t scratch_bytes, csg_stream_t stream);

/* ------------------------------------------------------------------------
 * SurfWarp: stencil feature operators (device).
 * Replace SurfaceStencilDevice's operators
 * (src/cat_surface_gpu/surface_stencil.py:282-644).  Neighbour lists are the
 * unique ascending 1-ring CSR of csg_mesh_neighbours; sums run in that order.
 * ---------------------------------------------------------------------- */

/* resample_vertices (282-306): out[i] = sum_k w[i][k] * vertices[indices[i][k]];
 * CSG_DTYPE_F32 sums float32-rounded float64 products, CSG_DTYPE_F64 sums in
 * float64. */
CSG_API int csg_feature_resample(int dtype, int n_out, const int32_t *indices, const double *weights,
                                 const void *vertices, void *out, csg_stream_t stream);

/* map_values_to_sheet (308-317), float64. */
CSG_API int csg_feature_sheet_map(int n_cells, const int32_t *indices, const double *weights, const double *values,
                                  double *out, csg_stream_t stream);

/* Scratch for the feature operators below. */
CSG_API size_t csg_feature_scratch_bytes(int n_points, int n_faces, int n_slots, int series);

/* Sum of the 3 n_faces edge lengths in float64 (for _edge_mean_distance, 347-356). */
CSG_API int csg_feature_edge_sum(int dtype, int n_faces, const int32_t *faces, const void *vertices, double *out_sum,
                                 void *scratch, size_t scratch_bytes, csg_stream_t stream);

/* smooth_geometry (372-388): `iterations` Jacobi heat steps, float32 out (must not overlap vertices). */
CSG_API int csg_feature_smooth_geometry(int n_points, const int32_t *nbr_off, const int32_t *nbr, const float *vertices,
                                        int iterations, float *out, void *scratch, size_t scratch_bytes,
                                        csg_stream_t stream);

/* smooth_values / smooth_values_many (390-476): `series` independent
 * smoothings of one value field (<= 16), sigma and iteration count per series
 * (host arrays); via_norm selects the single-FWHM distance form.
 * out [series][n_points], which must not overlap values (CSG_ERR_ARG). */
CSG_API int csg_feature_smooth_values(int n_points, const int32_t *nbr_off, const int32_t *nbr, int n_slots,
                                      int geometry_dtype, const void *geometry, const double *values, int series,
                                      const double *sigmas, const int32_t *iterations, int via_norm, double *out,
                                      void *scratch, size_t scratch_bytes, csg_stream_t stream);

/* vertex_normals (478-505); inc = per-vertex (face << 2 | corner) sorted by
 * (corner, face), inc_off [n_points + 1]. */
CSG_API int csg_feature_vertex_normals(int n_points, const int32_t *faces, const int32_t *inc_off, const int32_t *inc,
                                       const float *vertices, float *out, csg_stream_t stream);

/* ((smoothed - geometry) . normals) in float32, as float64 (curvature type 5, 512-515). */
CSG_API int csg_feature_normal_displacement(int n_points, const float *smoothed, const float *geometry,
                                            const float *normals, double *out, csg_stream_t stream);

/* curvature_type2 point values before smoothing (552-615), float64. */
CSG_API int csg_feature_curvature2(int n_points, const int32_t *nbr_off, const int32_t *nbr, const float *vertices,
                                   const float *normals, double *out, csg_stream_t stream);

/* (v - min) / (max - min) per row of `series` rows of n values. */
CSG_API int csg_feature_minmax(int n, int series, const double *values, double *out, void *scratch,
                               size_t scratch_bytes, csg_stream_t stream);

/* ------------------------------------------------------------------------
 * SurfWarp: resampling stencils (host, float64, threaded, deterministic).
 * Replaces the reference's stencil helper
 * (native/cat_surface_stencil_builder.c:107-170, 355-464) with the same
 * outputs: the resampling sphere's unit directions placed at
 * centre + r u (centre = per-axis min + max of the input points, r = 0.975 x
 * their mean length); surface barycentrics of each placed point under the
 * helper's closest-polygon rule (plane projection accepted within a 1e-3
 * parametric tolerance, else the nearer edge at the triangle's nearest
 * vertex; smallest candidate distance, lowest triangle index on ties); the
 * sphere points (the input interpolated there); sheet barycentrics of the
 * nx x ny cell centres on the unit-normalised sphere points; unit-sphere
 * points of the input vertices.  The resampling sphere (points + faces) is
 * the caller's (the helper's is 81,920 triangles).  normalize centres the
 * input on its vertex mean and projects it to unit length first. */
CSG_API int csg_stencil_build(const float *sphere, int n_sphere, const int32_t *sphere_faces, int n_sphere_faces,
                              const double *resampling_points, int n_points, const int32_t *resampling_faces,
                              int n_faces, int nx, int ny, int normalize, int threads, double *sphere_points_out,
                              int32_t *surface_indices_out, double *surface_weights_out, int32_t *sheet_indices_out,
                              double *sheet_weights_out, float *unit_points_out);

/* The same stencil built on the device (closest-point queries, grids and
 * scans on the GPU; the input preparation and sheet directions on the host),
 * bit-identical to csg_stencil_build.  Inputs and outputs are host arrays;
 * scratch is device memory of csg_stencil_scratch_bytes(); the call
 * synchronises `stream`.  CSG_ERR_UNSUPPORTED when a grid cell list would
 * exceed its capacity (triangles far larger than the grid cells), which the
 * host builder handles. */
CSG_API size_t csg_stencil_scratch_bytes(int n_sphere, int n_sphere_faces, int n_points, int n_faces, int nx, int ny);
CSG_API int csg_stencil_build_device(const float *sphere, int n_sphere, const int32_t *sphere_faces,
                                     int n_sphere_faces, const double *resampling_points, int n_points,
                                     const int32_t *resampling_faces, int n_faces, int nx, int ny, int normalize,
                                     double *sphere_points_out, int32_t *surface_indices_out,
                                     double *surface_weights_out, int32_t *sheet_indices_out,
                                     double *sheet_weights_out, float *unit_points_out, void *scratch,
                                     size_t scratch_bytes, csg_stream_t stream);

/* ------------------------------------------------------------------------
 * GIFTI payloads (host only; replaces the decode inside nibabel's GIFTI
 * reader that src/cat_surface_gpu/gpu_pipeline.py:52-71 read_gifti_mesh calls).
 * ------------------------------------------------------------------------ */

/* Decode one DataArray payload: `text` is its base64 text (whitespace allowed
 * anywhere, '=' padding only at the end), `gzip` 1 for GZipBase64Binary (a
 * zlib stream, Adler-32 checked) or 0 for Base64Binary.  `out` receives exactly
 * `out_bytes` bytes, the array's size from its header; a payload that decodes
 * to any other size is CSG_ERR_FORMAT, as is bad base64 or a corrupt or
 * truncated stream.  When `chunk_lengths` [n_chunks] gives the compressed
 * lengths of a stream deflated in raw chunks of `chunk_bytes` input bytes
 * (each ended by a sync flush, the last by the final block) and fits the
 * stream, the chunks inflate on up to 8 threads; an index that does not fit
 * is ignored and the stream inflates as one.  `adler32_out` (may be null)
 * receives the Adler-32 of the array's bytes (for a zlib stream, its verified
 * check value).  Holds no lock and touches no device. */
CSG_API int csg_gifti_decode(const char *text, size_t text_bytes, int gzip, const long long *chunk_lengths,
                             int n_chunks, long long chunk_bytes, void *out, size_t out_bytes,
                             unsigned int *adler32_out);

/* Synchronously read a persistent kernel's status word from its scratch. */
CSG_API int csg_read_status(const void *scratch, csg_stream_t stream, int *status, int *where);

#ifdef __cplusplus
}
#endif

#endif /* CATSURF_B200_H */
