/*
 * ORACLE -- test infrastructure only.  Nothing in the product path links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference leg of bench.py use it, as the checker.
 *
 * CPU restatement of CAT_Surf2Sphere's ordered area-smoothing sweeps as the
 * reference implements them:
 *
 *   - per-vertex update: src/cat_surface_gpu/surf2sphere.py:35-219
 *     (_areal_smoothing_kernel).  Each vertex moves to the area-weighted
 *     centroid of its incident faces; areas are clamped to [0, 1]
 *     (surf2sphere.py:190); total area <= 0 keeps the old position
 *     (surf2sphere.py:197-203).
 *   - "cat" mixed arithmetic (surf2sphere.py:54-215): float32 edges and
 *     cross product, float32 sum of squares, float64 sqrt / centre /
 *     accumulation / division, float32 store.
 *   - sphere projection every project_every sweeps:
 *     surf2sphere.py:222-280 (_normalize_points_kernel) and 1077-1092.
 *   - sweep driver: surf2sphere.py:1039-1092 -- sweeps 1 .. iterations-1,
 *     projection after sweep s when s % project_every == 0.
 *   - order: plain sequential Gauss-Seidel in vertex index order.  The
 *     reference's level groups (surface_stencil.py:94-109) are an exact
 *     re-scheduling of this order; incident faces are visited in ascending
 *     face id (surf2sphere.py:417-436, stable argsort).
 *
 * Floating-point expressions are written one rounding per operation and this
 * file is compiled with -ffp-contract=off, so the result is a deterministic
 * function of the IEEE-754 binary32/binary64 operations listed above.
 *
 * Arithmetic modes: 0 = "cat" mixed (default path), 1 = plain float32
 * ("fp32" arithmetic), 2 = float64 storage and arithmetic.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int build_incidence(int n, const int32_t *faces, int n_faces, int32_t **off_out, int32_t **inc_out)
{
    int32_t *off = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
    int32_t *inc = (int32_t *)malloc(sizeof(int32_t) * (size_t)(3 * n_faces + 1));
    int32_t *fill = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    if (!off || !inc || !fill) { free(off); free(inc); free(fill); return -1; }
    for (int f = 0; f < n_faces; ++f)
        for (int k = 0; k < 3; ++k) {
            int v = faces[3 * f + k];
            if (v < 0 || v >= n) { free(off); free(inc); free(fill); return -2; }
            off[v + 1]++;
        }
    for (int v = 0; v < n; ++v) off[v + 1] += off[v];
    for (int f = 0; f < n_faces; ++f)          /* ascending face id per vertex */
        for (int k = 0; k < 3; ++k) {
            int v = faces[3 * f + k];
            inc[off[v] + fill[v]++] = f;
        }
    free(fill);
    *off_out = off;
    *inc_out = inc;
    return 0;
}

static void update_cat(float *p, int v, const int32_t *faces, const int32_t *off, const int32_t *inc)
{
    double total = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int s = off[v]; s < off[v + 1]; ++s) {
        const int32_t *f = faces + 3 * inc[s];
        const float *a = p + 3 * f[0], *b = p + 3 * f[1], *c = p + 3 * f[2];
        float e0x = b[0] - a[0], e0y = b[1] - a[1], e0z = b[2] - a[2];
        float e1x = c[0] - a[0], e1y = c[1] - a[1], e1z = c[2] - a[2];
        float t0, t1;
        t0 = e0y * e1z; t1 = e0z * e1y; float cx = t0 - t1;
        t0 = e0z * e1x; t1 = e0x * e1z; float cy = t0 - t1;
        t0 = e0x * e1y; t1 = e0y * e1x; float cz = t0 - t1;
        float sq = cx * cx; t0 = cy * cy; sq = sq + t0; t0 = cz * cz; sq = sq + t0;
        double area = 0.5 * sqrt((double)sq);
        double mx = (((double)a[0] + (double)b[0]) + (double)c[0]) / 3.0;
        double my = (((double)a[1] + (double)b[1]) + (double)c[1]) / 3.0;
        double mz = (((double)a[2] + (double)b[2]) + (double)c[2]) / 3.0;
        area = area > 0.0 ? area : 0.0;
        area = area < 1.0 ? area : 1.0;
        total = total + area;
        double q;
        q = area * mx; wx = wx + q;
        q = area * my; wy = wy + q;
        q = area * mz; wz = wz + q;
    }
    if (total > 0.0) {
        double safe = total > 1.0e-20 ? total : 1.0e-20;
        p[3 * v + 0] = (float)(wx / safe);
        p[3 * v + 1] = (float)(wy / safe);
        p[3 * v + 2] = (float)(wz / safe);
    }
}

static void update_f32(float *p, int v, const int32_t *faces, const int32_t *off, const int32_t *inc)
{
    float total = 0.0f, wx = 0.0f, wy = 0.0f, wz = 0.0f;
    for (int s = off[v]; s < off[v + 1]; ++s) {
        const int32_t *f = faces + 3 * inc[s];
        const float *a = p + 3 * f[0], *b = p + 3 * f[1], *c = p + 3 * f[2];
        float e0x = b[0] - a[0], e0y = b[1] - a[1], e0z = b[2] - a[2];
        float e1x = c[0] - a[0], e1y = c[1] - a[1], e1z = c[2] - a[2];
        float t0, t1;
        t0 = e0y * e1z; t1 = e0z * e1y; float cx = t0 - t1;
        t0 = e0z * e1x; t1 = e0x * e1z; float cy = t0 - t1;
        t0 = e0x * e1y; t1 = e0y * e1x; float cz = t0 - t1;
        float sq = cx * cx; t0 = cy * cy; sq = sq + t0; t0 = cz * cz; sq = sq + t0;
        float area = 0.5f * sqrtf(sq);
        float mx = ((a[0] + b[0]) + c[0]) / 3.0f;
        float my = ((a[1] + b[1]) + c[1]) / 3.0f;
        float mz = ((a[2] + b[2]) + c[2]) / 3.0f;
        area = area > 0.0f ? area : 0.0f;
        area = area < 1.0f ? area : 1.0f;
        total = total + area;
        float q;
        q = area * mx; wx = wx + q;
        q = area * my; wy = wy + q;
        q = area * mz; wz = wz + q;
    }
    if (total > 0.0f) {
        float safe = total > 1.0e-20f ? total : 1.0e-20f;
        p[3 * v + 0] = wx / safe;
        p[3 * v + 1] = wy / safe;
        p[3 * v + 2] = wz / safe;
    }
}

static void update_f64(double *p, int v, const int32_t *faces, const int32_t *off, const int32_t *inc)
{
    double total = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int s = off[v]; s < off[v + 1]; ++s) {
        const int32_t *f = faces + 3 * inc[s];
        const double *a = p + 3 * f[0], *b = p + 3 * f[1], *c = p + 3 * f[2];
        double e0x = b[0] - a[0], e0y = b[1] - a[1], e0z = b[2] - a[2];
        double e1x = c[0] - a[0], e1y = c[1] - a[1], e1z = c[2] - a[2];
        double t0, t1;
        t0 = e0y * e1z; t1 = e0z * e1y; double cx = t0 - t1;
        t0 = e0z * e1x; t1 = e0x * e1z; double cy = t0 - t1;
        t0 = e0x * e1y; t1 = e0y * e1x; double cz = t0 - t1;
        double sq = cx * cx; t0 = cy * cy; sq = sq + t0; t0 = cz * cz; sq = sq + t0;
        double area = 0.5 * sqrt(sq);
        double mx = ((a[0] + b[0]) + c[0]) / 3.0;
        double my = ((a[1] + b[1]) + c[1]) / 3.0;
        double mz = ((a[2] + b[2]) + c[2]) / 3.0;
        area = area > 0.0 ? area : 0.0;
        area = area < 1.0 ? area : 1.0;
        total = total + area;
        double q;
        q = area * mx; wx = wx + q;
        q = area * my; wy = wy + q;
        q = area * mz; wz = wz + q;
    }
    if (total > 0.0) {
        double safe = total > 1.0e-20 ? total : 1.0e-20;
        p[3 * v + 0] = wx / safe;
        p[3 * v + 1] = wy / safe;
        p[3 * v + 2] = wz / safe;
    }
}

static void project_cat(float *p, int n, double radius)
{
    for (int v = 0; v < n; ++v) {
        float x = p[3 * v], y = p[3 * v + 1], z = p[3 * v + 2];
        float sq = x * x, t = y * y; sq = sq + t; t = z * z; sq = sq + t;
        double norm = sqrt((double)sq);
        double scale = radius / (norm > 1.0e-20 ? norm : 1.0e-20);
        p[3 * v + 0] = (float)((double)x * scale);
        p[3 * v + 1] = (float)((double)y * scale);
        p[3 * v + 2] = (float)((double)z * scale);
    }
}

static void project_f32(float *p, int n, float radius)
{
    for (int v = 0; v < n; ++v) {
        float x = p[3 * v], y = p[3 * v + 1], z = p[3 * v + 2];
        float sq = x * x, t = y * y; sq = sq + t; t = z * z; sq = sq + t;
        float norm = sqrtf(sq);
        float scale = radius / (norm > 1.0e-20f ? norm : 1.0e-20f);
        p[3 * v + 0] = x * scale;
        p[3 * v + 1] = y * scale;
        p[3 * v + 2] = z * scale;
    }
}

static void project_f64(double *p, int n, double radius)
{
    for (int v = 0; v < n; ++v) {
        double x = p[3 * v], y = p[3 * v + 1], z = p[3 * v + 2];
        double sq = x * x, t = y * y; sq = sq + t; t = z * z; sq = sq + t;
        double norm = sqrt(sq);
        double scale = radius / (norm > 1.0e-20 ? norm : 1.0e-20);
        p[3 * v + 0] = x * scale;
        p[3 * v + 1] = y * scale;
        p[3 * v + 2] = z * scale;
    }
}

/* points: float32 [n,3] for modes 0/1, float64 [n,3] for mode 2 (in place).
 * Returns 0 on success, negative on bad arguments. */
int oracle_areal_sweeps(void *points, int n, const int32_t *faces, int n_faces, int iterations,
                        int project_every, double radius, int mode)
{
    if (n < 1 || n_faces < 0 || iterations < 1 || project_every < 0 || mode < 0 || mode > 2) return -1;
    int32_t *off = NULL, *inc = NULL;
    int rc = build_incidence(n, faces, n_faces, &off, &inc);
    if (rc) return rc;
    for (int it = 1; it < iterations; ++it) {
        if (mode == 0) {
            float *p = (float *)points;
            for (int v = 0; v < n; ++v) update_cat(p, v, faces, off, inc);
            if (project_every > 0 && it % project_every == 0) project_cat(p, n, radius);
        } else if (mode == 1) {
            float *p = (float *)points;
            for (int v = 0; v < n; ++v) update_f32(p, v, faces, off, inc);
            if (project_every > 0 && it % project_every == 0) project_f32(p, n, (float)radius);
        } else {
            double *p = (double *)points;
            for (int v = 0; v < n; ++v) update_f64(p, v, faces, off, inc);
            if (project_every > 0 && it % project_every == 0) project_f64(p, n, radius);
        }
    }
    free(off);
    free(inc);
    return 0;
}

/* Dependency levels: level(v) = 1 + max level of lower-index neighbours, 0 if
 * none (surface_stencil.py:94-109).  Neighbours are the vertices sharing a
 * triangle edge.  levels: int32 [n] output. Returns the level count. */
int oracle_dependency_levels(int n, const int32_t *faces, int n_faces, int32_t *levels)
{
    int32_t *off = NULL, *inc = NULL;
    if (build_incidence(n, faces, n_faces, &off, &inc)) return -1;
    int count = 0;
    for (int v = 0; v < n; ++v) {
        int level = 0;
        for (int s = off[v]; s < off[v + 1]; ++s) {
            const int32_t *f = faces + 3 * inc[s];
            for (int k = 0; k < 3; ++k) {
                int u = f[k];
                if (u < v && levels[u] + 1 > level) level = levels[u] + 1;
            }
        }
        levels[v] = level;
        if (level + 1 > count) count = level + 1;
    }
    free(off);
    free(inc);
    return count;
}
