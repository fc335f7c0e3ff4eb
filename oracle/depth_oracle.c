/* ORACLE (test infrastructure): C restatement of the depth-potential rotation
 * feature, src/cat_surface_gpu/rotation_feature.py.
 *
 *   depth_face_terms     _stable_normals 37-74, _mixed_voronoi_areas 77-128,
 *                        _system_entries 131-171 (per-face quantities)
 *   od_depth_setup       the per-vertex scatters (index_add_) in the reference's
 *                        entry order, the system rows, the Laplacian, the mean
 *                        curvature, rhs and diagonal (189-230 / 253-290)
 *   od_depth_sor         _solve_depth_potential_colored_sor 253-317
 *   od_depth_pcg         _solve_depth_potential_cg 189-250
 *
 * Arithmetic is float64 with one rounding per operation (-ffp-contract=off),
 * except where the reference's torch CPU kernels fuse: vector_norm accumulates
 * fma(x_i, x_i, acc) and linalg.cross forms fma(a, b, -(c d)).  Elementwise
 * dot products over 3 components are ((x0 y0 + x1 y1) + x2 y2).
 *
 * Row order.  index_add_ on the CPU adds entries in order, so row v of the
 * system is: the diagonal entries of the faces where v is corner 0, 1, 2 (each
 * in face order), then the off-diagonal blocks (i0,i1) (i1,i0) (i1,i2) (i2,i1)
 * (i0,i2) (i2,i0), then alpha * area.  With the incidences of v sorted by
 * (corner, face) that is: all incidences, corner-0 ones, corner-1 ones twice,
 * corner-2 ones, corner-0 ones, corner-2 ones.
 *
 * Whole-vector sums (the mean-curvature offset, norms, CG's dot products) use
 * one fixed blocked order -- sequential runs of 256 terms, run sums r folded
 * into 32 lanes (lane l takes runs l, l + 32, ...), then the lanes pairwise
 * (16, 8, 4, 2, 1) -- which the device kernels use as well; torch's own
 * reduction order differs, so against the reference those agree to rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define RUN 256
static const double EPS = 2.220446049250313080847263336181640625e-16;

static double clamp_eps(double x) { return x < EPS ? EPS : x; } /* torch clamp_min keeps NaN */
static double dot3(const double *a, const double *b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
static double norm3(const double *a) { return sqrt(fma(a[2], a[2], fma(a[1], a[1], a[0] * a[0]))); }
static void cross3(const double *a, const double *b, double *o) {
    o[0] = fma(a[1], b[2], -(a[2] * b[1]));
    o[1] = fma(a[2], b[0], -(a[0] * b[2]));
    o[2] = fma(a[0], b[1], -(a[1] * b[0]));
}

/* the blocked sum of terms t[0..n) */
double od_blocked_sum(const double *t, int64_t n) {
    int64_t runs = (n + RUN - 1) / RUN;
    double lane[32];
    for (int l = 0; l < 32; ++l) lane[l] = 0.0;
    for (int64_t r = 0; r < runs; ++r) {
        double s = 0.0;
        for (int64_t i = r * RUN; i < n && i < (r + 1) * RUN; ++i) s = s + t[i];
        lane[r % 32] = lane[r % 32] + s;
    }
    for (int off = 16; off >= 1; off >>= 1)
        for (int l = 0; l < off; ++l) lane[l] = lane[l] + lane[l + off];
    return lane[0];
}

/* per face: tn[3], w[3] (stable normals), contribution[3] (mixed Voronoi areas),
 * d23, d13, d12 (system) -- 12 doubles */
static void depth_face_terms(const float *pts, const int32_t *faces, int nf, double *rec) {
    for (int f = 0; f < nf; ++f) {
        double p[3][3];
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) p[k][c] = (double)pts[3 * (int64_t)faces[3 * f + k] + c];
        double v1[3], v2[3], v3[3], u1[3], u2[3], u3[3];
        for (int c = 0; c < 3; ++c) {
            v1[c] = p[1][c] - p[0][c];
            v2[c] = p[2][c] - p[1][c];
            v3[c] = p[0][c] - p[2][c];
        }
        double n1 = clamp_eps(norm3(v1)), n2 = clamp_eps(norm3(v2)), n3 = clamp_eps(norm3(v3));
        for (int c = 0; c < 3; ++c) {
            u1[c] = v1[c] / n1;
            u2[c] = v2[c] / n2;
            u3[c] = v3[c] / n3;
        }
        double c31[3], c23[3], c12[3];
        cross3(u3, u1, c31);
        cross3(u2, u3, c23);
        cross3(u1, u2, c12);
        double m31 = clamp_eps(norm3(c31)), m23 = clamp_eps(norm3(c23)), m12 = clamp_eps(norm3(c12));
        double *r = rec + 12 * (int64_t)f;
        for (int c = 0; c < 3; ++c) r[c] = c12[c] / m12;
        r[3] = (1.0 - dot3(u3, u1)) / m31;
        r[4] = (1.0 - dot3(u1, u2)) / m12;
        r[5] = (1.0 - dot3(u2, u3)) / m23;
        double cr[3];
        cross3(v1, v2, cr);
        double area = clamp_eps(norm3(cr));
        double d31 = dot3(v3, v1), d12 = dot3(v1, v2), d23 = dot3(v2, v3);
        int bad0 = d31 > 0.0, bad1 = d12 > 0.0, bad2 = d23 > 0.0, bad = bad0 || bad1 || bad2;
        double l1 = dot3(v1, v1), l2 = dot3(v2, v2), l3 = dot3(v3, v3), d13 = dot3(v1, v3);
        double w0 = l3 * d12 + l1 * d23, w1 = l2 * d13 + l1 * d23, w2 = l2 * d13 + l3 * d12;
        double e = 0.125 * area;
        double con[3];
        if (bad) {
            con[0] = e + (bad0 ? e : 0.0);
            con[1] = e + (bad1 ? e : 0.0);
            con[2] = e + (bad2 ? e : 0.0);
        } else {
            con[0] = -0.125 * w0 / area + 0.0;
            con[1] = -0.125 * w1 / area + 0.0;
            con[2] = -0.125 * w2 / area + 0.0;
        }
        r[6] = con[0];
        r[7] = con[1];
        r[8] = con[2];
        r[9] = d23 / area;
        r[10] = d13 / area;
        r[11] = d12 / area;
    }
}

/* Row v's entries in the reference's order (see the file comment); returns the count. */
static int row_entries(int v, const int32_t *faces, const int32_t *inc_off, const int32_t *inc, const double *rec,
                       double alpha, double area, int32_t *col, double *val) {
    int m = 0;
    const int b = inc_off[v], e = inc_off[v + 1];
    for (int k = b; k < e; ++k) {
        const int f = inc[k] >> 2, corner = inc[k] & 3;
        const double *r = rec + 12 * (int64_t)f;
        const double d23 = r[9], d13 = r[10], d12 = r[11];
        col[m] = v;
        val[m++] = corner == 0 ? -0.5 * (d23 + d12) : (corner == 1 ? -0.5 * (d13 + d23) : -0.5 * (d12 + d13));
    }
    /* block: rows corner, column corner, value slot (9 d23, 10 d13, 11 d12) */
    static const int blocks[6][3] = {{0, 1, 9}, {1, 0, 9}, {1, 2, 10}, {2, 1, 10}, {0, 2, 11}, {2, 0, 11}};
    for (int q = 0; q < 6; ++q)
        for (int k = b; k < e; ++k) {
            const int f = inc[k] >> 2, corner = inc[k] & 3;
            if (corner != blocks[q][0]) continue;
            col[m] = faces[3 * f + blocks[q][1]];
            val[m++] = 0.5 * rec[12 * (int64_t)f + blocks[q][2]];
        }
    if (alpha != 0.0) {
        col[m] = v;
        val[m++] = alpha * area;
    }
    return m;
}

/* Geometry, system and right-hand side.  row_off[n+1], col/val[3 * inc_off[n] + n]
 * (rows of 3 deg + 1 entries; the last is alpha * area), diag[n], rhs[n];
 * returns rhs_norm = max(|rhs|, eps) through *rhs_norm. */
int od_depth_setup(const float *pts, int n, const int32_t *faces, int nf, const int32_t *inc_off, const int32_t *inc,
                   double alpha, double *normals, double *areas, int32_t *row_off, int32_t *col, double *val,
                   double *diag, double *rhs, double *rhs_norm) {
    if (alpha == 0.0) return -1;
    double *rec = malloc(sizeof(double) * 12 * (size_t)nf);
    double *mc = malloc(sizeof(double) * (size_t)n);
    double *terms = malloc(sizeof(double) * (size_t)n);
    if (!rec || !mc || !terms) return -2;
    depth_face_terms(pts, faces, nf, rec);
    row_off[0] = 0;
    for (int v = 0; v < n; ++v) {
        double acc[3] = {0.0, 0.0, 0.0}, a = 0.0;
        for (int k = inc_off[v]; k < inc_off[v + 1]; ++k) {
            const int f = inc[k] >> 2, corner = inc[k] & 3;
            const double *r = rec + 12 * (int64_t)f;
            for (int c = 0; c < 3; ++c) acc[c] = acc[c] + r[c] * r[3 + corner];
            a = a + r[6 + corner];
        }
        const double nn = clamp_eps(norm3(acc));
        double nv[3];
        for (int c = 0; c < 3; ++c) nv[c] = acc[c] / nn;
        if (!isfinite(a) || a == 0.0) a = 1.0;
        if (normals)
            for (int c = 0; c < 3; ++c) normals[3 * (int64_t)v + c] = nv[c];
        areas[v] = a;
        const int b = row_off[v];
        const int m = row_entries(v, faces, inc_off, inc, rec, alpha, a, col + b, val + b);
        row_off[v + 1] = b + m;
        double d = 0.0, lap[3] = {0.0, 0.0, 0.0};
        for (int k = b; k < b + m; ++k) d = d + (col[k] == v ? val[k] : 0.0);
        for (int k = b; k < b + m - 1; ++k) /* the Laplacian has no alpha entry */
            for (int c = 0; c < 3; ++c) lap[c] = lap[c] + val[k] * (double)pts[3 * (int64_t)col[k] + c];
        for (int c = 0; c < 3; ++c) lap[c] = lap[c] * 2.0;
        diag[v] = clamp_eps(d);
        double h = 0.5 * dot3(lap, nv) / a;
        mc[v] = isfinite(h) ? h : 0.0;
    }
    for (int v = 0; v < n; ++v) terms[v] = mc[v] * areas[v];
    const double factor = od_blocked_sum(terms, n) / od_blocked_sum(areas, n);
    for (int v = 0; v < n; ++v) rhs[v] = (mc[v] - factor) * areas[v];
    for (int v = 0; v < n; ++v) terms[v] = rhs[v] * rhs[v];
    *rhs_norm = clamp_eps(sqrt(od_blocked_sum(terms, n)));
    free(rec);
    free(mc);
    free(terms);
    return 0;
}

static double row_dot(int v, const int32_t *row_off, const int32_t *col, const double *val, const double *x) {
    double s = 0.0;
    for (int k = row_off[v]; k < row_off[v + 1]; ++k) s = s + val[k] * x[col[k]];
    return s;
}

static double residual_norm(int n, const int32_t *row_off, const int32_t *col, const double *val, const double *rhs,
                            const double *x, double *terms) {
    for (int v = 0; v < n; ++v) {
        const double r = rhs[v] - row_dot(v, row_off, col, val, x);
        terms[v] = r * r;
    }
    return sqrt(od_blocked_sum(terms, n));
}

int od_depth_sor(int n, const int32_t *row_off, const int32_t *col, const double *val, const double *diag,
                 const double *rhs, double rhs_norm, const int32_t *colour_off, const int32_t *members, int n_colours,
                 int max_iter, double relaxation, double *x, double *residual) {
    double *partial = malloc(sizeof(double) * (size_t)n);
    if (!partial) return -2;
    for (int v = 0; v < n; ++v) x[v] = 0.0;
    for (int it = 0; it < max_iter; ++it)
        for (int c = 0; c < n_colours; ++c) {
            for (int k = colour_off[c]; k < colour_off[c + 1]; ++k)
                partial[k - colour_off[c]] = row_dot(members[k], row_off, col, val, x);
            for (int k = colour_off[c]; k < colour_off[c + 1]; ++k) {
                const int v = members[k];
                x[v] = x[v] + relaxation * (rhs[v] - partial[k - colour_off[c]]) / diag[v];
            }
        }
    *residual = residual_norm(n, row_off, col, val, rhs, x, partial) / rhs_norm;
    free(partial);
    return 0;
}

int od_depth_pcg(int n, const int32_t *row_off, const int32_t *col, const double *val, const double *diag,
                 const double *rhs, double rhs_norm, int max_iter, double tolerance, double *x, int *iterations,
                 double *residual) {
    double *r = malloc(sizeof(double) * (size_t)n), *z = malloc(sizeof(double) * (size_t)n);
    double *p = malloc(sizeof(double) * (size_t)n), *ap = malloc(sizeof(double) * (size_t)n);
    double *t = malloc(sizeof(double) * (size_t)n);
    if (!r || !z || !p || !ap || !t) return -2;
    for (int v = 0; v < n; ++v) x[v] = 0.0;
    for (int v = 0; v < n; ++v) r[v] = rhs[v] - row_dot(v, row_off, col, val, x);
    for (int v = 0; v < n; ++v) t[v] = r[v] * r[v];
    double rel = sqrt(od_blocked_sum(t, n)) / rhs_norm;
    int its = 0;
    if (!(rel <= tolerance)) {
        for (int v = 0; v < n; ++v) {
            z[v] = r[v] / diag[v];
            p[v] = z[v];
            t[v] = r[v] * z[v];
        }
        double rho = od_blocked_sum(t, n);
        for (int it = 1; it <= max_iter; ++it) {
            for (int v = 0; v < n; ++v) {
                ap[v] = row_dot(v, row_off, col, val, p);
                t[v] = p[v] * ap[v];
            }
            const double step = rho / od_blocked_sum(t, n);
            for (int v = 0; v < n; ++v) {
                x[v] = x[v] + step * p[v];
                r[v] = r[v] - step * ap[v];
                t[v] = r[v] * r[v];
            }
            rel = sqrt(od_blocked_sum(t, n)) / rhs_norm;
            its = it;
            if (rel <= tolerance) break;
            for (int v = 0; v < n; ++v) {
                z[v] = r[v] / diag[v];
                t[v] = r[v] * z[v];
            }
            const double new_rho = od_blocked_sum(t, n);
            const double beta = new_rho / rho;
            for (int v = 0; v < n; ++v) p[v] = z[v] + beta * p[v];
            rho = new_rho;
        }
    }
    *iterations = its;
    *residual = rel;
    free(r);
    free(z);
    free(p);
    free(ap);
    free(t);
    return 0;
}
