/*
 * ORACLE -- test infrastructure only.  Nothing in the product path links,
 * loads or calls this file; only tests/ and the CPU legs of bench.py use it,
 * as the checker.
 *
 * CPU restatement of CAT_Surf2Sphere's stages 1-5 (low_smooth, inflate,
 * very_inflate, high_smooth, ellipsoid) as the reference describes them in
 * src/cat_surface_gpu/surf2sphere.py:
 *
 *   - stage table and iteration scaling: 758-814 (factor F / 350,000 for
 *     meshes above 350,000 faces);
 *   - one stage: 632-713 (_run_inflate_surface_stage_cuda): keep the stage's
 *     input as the reference geometry, centre on the vertex mean, then for
 *     cycle 0..cycles-1: `iterations - 1` distance-smoothing passes, the
 *     inflation scale 1 + (factor - 1) (1 - |p / extent|), the distortion
 *     selection, and `finger_iterations - 1` distance-smoothing passes over
 *     the selected vertices;
 *   - distance smoothing: 283-397 (_distance_smoothing_kernel): each vertex
 *     moves to (1 - s) p + s (sum_j d_j q_j / sum_j d_j) with d_j the L1
 *     distance to neighbour j; vertices of degree <= 1 stay;
 *   - face and vertex areas: 474-492; distortion selection: 573-629.
 *
 * Order: plain sequential Gauss-Seidel in vertex index order (the upstream
 * binary's order; the reference's Triton path re-orders by colour).
 * Arithmetic: float32 storage, float64 arithmetic, one rounding per
 * operation (-ffp-contract=off).  Sums over all vertices or faces (the
 * centre, the surface area) are blocked: sequential within runs of
 * BLOCK_SUM consecutive elements, then sequentially over the runs -- the
 * order the GPU kernels use.  Against the upstream binary's stage 1-5
 * outputs this ordering and precision agree to ~1e-5 where the colour order
 * disagrees by ~1e-1.
 *
 * Neighbour lists: the unique ascending 1-ring (surface_stencil.py:36-66).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define BLOCK_SUM 256

/* sum of x[0 .. n), blocked as described above */
static double blocked_sum(const double *x, int n)
{
    double total = 0.0;
    for (int b = 0; b < n; b += BLOCK_SUM) {
        double part = 0.0;
        for (int i = b; i < n && i < b + BLOCK_SUM; ++i) part = part + x[i];
        total = total + part;
    }
    return total;
}

typedef struct {
    int cycles;
    double strength;
    int iterations;
    double inflation;
    double threshold;
    double finger_strength;
    int finger_iterations;
} Stage;

static const Stage STAGES[5] = {
    {1, 0.2, 50, 1.0, 3.0, 1.0, 0},  /* low_smooth */
    {2, 1.0, 30, 1.4, 3.0, 1.0, 30}, /* inflate */
    {4, 1.0, 30, 1.1, 3.0, 1.0, 0},  /* very_inflate */
    {6, 1.0, 60, 1.6, 3.0, 1.0, 60}, /* high_smooth */
    {6, 1.0, 50, 1.4, 4.0, 1.0, 60}, /* ellipsoid */
};

/* One Gauss-Seidel distance-smoothing pass; `selected` may be NULL (all). */
static void smooth_pass(float *p, int n, const int32_t *off, const int32_t *nb, double strength,
                        const unsigned char *selected)
{
    const double inv = 1.0 - strength;
    for (int v = 0; v < n; ++v) {
        const int b = off[v], e = off[v + 1];
        if (e - b <= 1) continue;
        if (selected && !selected[v]) continue;
        const double ox = p[3 * v], oy = p[3 * v + 1], oz = p[3 * v + 2];
        double total = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
        for (int k = b; k < e; ++k) {
            const int u = nb[k];
            const double qx = p[3 * u], qy = p[3 * u + 1], qz = p[3 * u + 2];
            const double d = (fabs(qx - ox) + fabs(qy - oy)) + fabs(qz - oz);
            total = total + d;
            if (d > 0.0) {
                wx = wx + d * qx;
                wy = wy + d * qy;
                wz = wz + d * qz;
            }
        }
        double cx, cy, cz;
        if (total > 0.0) {
            cx = ox * inv + (wx / total) * strength;
            cy = oy * inv + (wy / total) * strength;
            cz = oz * inv + (wz / total) * strength;
        } else {
            cx = ox * inv;
            cy = oy * inv;
            cz = oz * inv;
        }
        p[3 * v] = (float)cx;
        p[3 * v + 1] = (float)cy;
        p[3 * v + 2] = (float)cz;
    }
}

/* Face areas (blocked sum returned) and vertex areas (a third of each face,
 * per column in face order, like three index_add passes). */
static double areas(const float *p, int n, const int32_t *faces, int nf, double *vertex_area)
{
    memset(vertex_area, 0, sizeof(double) * (size_t)n);
    double *fa = (double *)malloc(sizeof(double) * (size_t)nf);
    for (int f = 0; f < nf; ++f) {
        const float *a = p + 3 * faces[3 * f], *b = p + 3 * faces[3 * f + 1], *c = p + 3 * faces[3 * f + 2];
        const double e0x = (double)b[0] - a[0], e0y = (double)b[1] - a[1], e0z = (double)b[2] - a[2];
        const double e1x = (double)c[0] - a[0], e1y = (double)c[1] - a[1], e1z = (double)c[2] - a[2];
        const double cx = e0y * e1z - e0z * e1y, cy = e0z * e1x - e0x * e1z, cz = e0x * e1y - e0y * e1x;
        double area = 0.5 * sqrt((cx * cx + cy * cy) + cz * cz);
        if (isnan(area)) area = 0.0;
        fa[f] = area;
    }
    const double surface = blocked_sum(fa, nf);
    for (int k = 0; k < 3; ++k)
        for (int f = 0; f < nf; ++f) vertex_area[faces[3 * f + k]] += fa[f] / 3.0;
    free(fa);
    return surface;
}

static void selection(const float *p, const float *ref, int n, const int32_t *off, const int32_t *nb,
                      const double *cur_area, const double *ref_area, double surface_ratio, double threshold,
                      double *comp, unsigned char *selected)
{
    for (int v = 0; v < n; ++v) {
        double max_linear = 0.0;
        for (int k = off[v]; k < off[v + 1]; ++k) {
            const int u = nb[k];
            const double cx = (double)p[3 * u] - p[3 * v], cy = (double)p[3 * u + 1] - p[3 * v + 1],
                         cz = (double)p[3 * u + 2] - p[3 * v + 2];
            const double rx = (double)ref[3 * u] - ref[3 * v], ry = (double)ref[3 * u + 1] - ref[3 * v + 1],
                         rz = (double)ref[3 * u + 2] - ref[3 * v + 2];
            const double cd = sqrt((cx * cx + cy * cy) + cz * cz), rd = sqrt((rx * rx + ry * ry) + rz * rz);
            const double ratio = rd > 0.0 ? cd / rd : 0.0;
            if (ratio > max_linear) max_linear = ratio;
        }
        double area_ratio;
        if (cur_area[v] > 0.0) area_ratio = ref_area[v] / cur_area[v];
        else area_ratio = ref_area[v] != 0.0 ? 10000.0 : 1.0;
        if (area_ratio < 1.0e-8) area_ratio = 1.0e-8;
        comp[v] = max_linear * area_ratio * surface_ratio;
    }
    for (int v = 0; v < n; ++v) {
        double sum = comp[v];
        for (int k = off[v]; k < off[v + 1]; ++k) sum = sum + comp[nb[k]];
        selected[v] = (sum / (double)(off[v + 1] - off[v] + 1)) > threshold;
    }
}

/* Stages 1..stop_at (1..5) in place on float32 points [n][3]. */
int oracle_surf2sphere_preprocess(float *points, int n, const int32_t *faces, int nf, const int32_t *nb_off,
                                  const int32_t *nb, int stop_at)
{
    if (!points || !faces || !nb_off || !nb || n < 4 || nf < 4 || stop_at < 1 || stop_at > 5) return -1;
    const double factor = nf > 350000 ? (double)nf / 350000.0 : 1.0;
    float *ref = (float *)malloc(sizeof(float) * 3 * (size_t)n);
    double *ref_area = (double *)malloc(sizeof(double) * (size_t)n);
    double *cur_area = (double *)malloc(sizeof(double) * (size_t)n);
    double *comp = (double *)malloc(sizeof(double) * (size_t)n);
    unsigned char *selected = (unsigned char *)malloc((size_t)n);
    if (!ref || !ref_area || !cur_area || !comp || !selected) {
        free(ref); free(ref_area); free(cur_area); free(comp); free(selected);
        return -2;
    }
    for (int s = 0; s < stop_at; ++s) {
        const Stage st = STAGES[s];
        const int iterations = (int)nearbyint(factor * st.iterations); /* round half to even, like round() */
        const int finger = (int)nearbyint(factor * st.finger_iterations);
        memcpy(ref, points, sizeof(float) * 3 * (size_t)n);
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        double mean[3], extent[3];
        for (int k = 0; k < 3; ++k) {
            for (int v = 0; v < n; ++v) {
                const double x = ref[3 * v + k];
                if (x < lo[k]) lo[k] = x;
                if (x > hi[k]) hi[k] = x;
                comp[v] = x;
            }
            mean[k] = blocked_sum(comp, n) / n;
            extent[k] = hi[k] - lo[k];
            if (extent[k] < 1.0e-20) extent[k] = 1.0e-20;
        }
        for (int v = 0; v < n; ++v)
            for (int k = 0; k < 3; ++k) points[3 * v + k] = (float)((double)points[3 * v + k] - mean[k]);
        const double ref_surface = areas(ref, n, faces, nf, ref_area);
        const double delta = st.inflation - 1.0;
        for (int cycle = 0; cycle < st.cycles; ++cycle) {
            for (int it = 1; it < iterations; ++it) smooth_pass(points, n, nb_off, nb, st.strength, NULL);
            for (int v = 0; v < n; ++v) {
                const double x = points[3 * v] / extent[0], y = points[3 * v + 1] / extent[1],
                             z = points[3 * v + 2] / extent[2];
                const double scale = 1.0 + delta * (1.0 - sqrt((x * x + y * y) + z * z));
                for (int k = 0; k < 3; ++k) points[3 * v + k] = (float)((double)points[3 * v + k] * scale);
            }
            if (finger > 0) {
                const double surface = areas(points, n, faces, nf, cur_area);
                const double ratio = surface / (ref_surface > 1.0e-30 ? ref_surface : 1.0e-30);
                selection(points, ref, n, nb_off, nb, cur_area, ref_area, ratio, st.threshold, comp, selected);
                for (int it = 1; it < finger; ++it)
                    smooth_pass(points, n, nb_off, nb, st.finger_strength, selected);
            }
        }
    }
    free(ref); free(ref_area); free(cur_area); free(comp); free(selected);
    return 0;
}
