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

#define CSG_ARITH_CAT 0  /* float32 storage, CAT mixed float32/float64 arithmetic */
#define CSG_ARITH_FP32 1 /* float32 storage and arithmetic */
#define CSG_ARITH_FP64 2 /* float64 storage and arithmetic */

CSG_API const char *csg_last_error(void);
CSG_API int csg_abi_version(void);

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

/* level(v) = 1 + max level of lower-index neighbours (0 if none).
 * Replaces _build_ordered_dependency_groups
 * (src/cat_surface_gpu/surface_stencil.py:94-109).  Returns the level count. */
CSG_API int csg_dependency_levels(int n_vertices, const int32_t *nbr_off, const int32_t *nbr, int32_t *levels);

/* Greedy colouring in vertex order.  Replaces _build_color_groups
 * (src/cat_surface_gpu/surface_stencil.py:69-91).  Returns the colour count. */
CSG_API int csg_greedy_colours(int n_vertices, const int32_t *nbr_off, const int32_t *nbr, int32_t *colours);

/* Wavefront plan for the ordered sweeps (host).
 * Vertex v of sweep s runs at wavefront step s * level_stride + level(v);
 * level_stride = 1 + max over edges (v < w) of level(w) - level(v), which
 * keeps exactly the sequential Gauss-Seidel reads (lower neighbours of the
 * current sweep, higher neighbours of the previous one).
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
CSG_API size_t csg_areal_scratch_bytes(int n_vertices, int arithmetic);

CSG_API int csg_areal_sweeps(void *points, int n_vertices, const int32_t *slot_off, const int32_t *slot_tri,
                     const int32_t *order, const int32_t *level_begin, const int32_t *level_end, int n_levels,
                     int level_stride, int max_degree, int iterations, int project_every, double radius, int arithmetic, void *scratch,
                     size_t scratch_bytes, int n_ctas, int threads_per_cta, int lanes_per_vertex, double timeout_s,
                     csg_stream_t stream);

/* Self-test of the bounded device-side wait (no reference counterpart): a
 * 2-CTA cooperative grid waits on a barrier that expects one arrival more
 * than the grid has; the wait gives up after timeout_s (<= 10 s) and records
 * CSG_ERR_TIMEOUT in scratch's status word.  Exercises the timeout path
 * without faulting or hanging the GPU; the context stays usable. */
CSG_API int csg_selftest_barrier_timeout(void *scratch, size_t scratch_bytes, double timeout_s, csg_stream_t stream);

/* Synchronously read a persistent kernel's status word from its scratch. */
CSG_API int csg_read_status(const void *scratch, csg_stream_t stream, int *status, int *where);

#ifdef __cplusplus
}
#endif

#endif /* CATSURF_B200_H */
