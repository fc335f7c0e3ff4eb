// Spherical resampling stencils (host C++, float64, deterministic, threaded).
//
// Builds the same stencil the reference's helper writes
// (native/cat_surface_stencil_builder.c:172-464 in the reference project):
//   * sphere points: the resampling sphere's points moved onto the input
//     sphere (closest point on the input's triangles);
//   * surface barycentrics: for every resampling-sphere point scaled to
//     0.975 x the mean input radius, the closest input triangle and the
//     barycentric weights of the closest point -- indices refer to the
//     surface (same topology as the sphere);
//   * sheet barycentrics: for every sheet cell centre (u, v) =
//     ((x + 0.5) / nx, (y + 0.5) / ny) mapped to the unit point
//     (sin(pi v) cos(2 pi u), sin(pi v) sin(2 pi u), cos(pi v)), the closest
//     triangle of the unit-normalised sphere points;
//   * unit-sphere points of the input vertices.
// The resampling sphere (points + faces) is supplied by the caller.  Closest
// points are exact: a uniform grid over the target triangles is searched in
// growing shells of cells until no unvisited cell can hold a closer point;
// ties keep the lowest triangle index.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/catsurf_b200.h"
#include "errors.h"

namespace {

struct V3 {
    double x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// Closest point of p on triangle abc with its barycentric weights (Voronoi
// region classification of the point against the triangle's features;
// Ericson, Real-Time Collision Detection, 5.1.5).
double closest_on_triangle(V3 p, V3 a, V3 b, V3 c, double w[3]) {
    const V3 ab = b - a, ac = c - a, ap = p - a;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    V3 q;
    if (d1 <= 0.0 && d2 <= 0.0) {
        w[0] = 1; w[1] = 0; w[2] = 0;
        q = a;
    } else {
        const V3 bp = p - b;
        const double d3 = dot(ab, bp), d4 = dot(ac, bp);
        if (d3 >= 0.0 && d4 <= d3) {
            w[0] = 0; w[1] = 1; w[2] = 0;
            q = b;
        } else {
            const double vc = d1 * d4 - d3 * d2;
            if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
                const double t = d1 / (d1 - d3);
                w[0] = 1 - t; w[1] = t; w[2] = 0;
                q = a + t * ab;
            } else {
                const V3 cp = p - c;
                const double d5 = dot(ab, cp), d6 = dot(ac, cp);
                if (d6 >= 0.0 && d5 <= d6) {
                    w[0] = 0; w[1] = 0; w[2] = 1;
                    q = c;
                } else {
                    const double vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
                        const double t = d2 / (d2 - d6);
                        w[0] = 1 - t; w[1] = 0; w[2] = t;
                        q = a + t * ac;
                    } else {
                        const double va = d3 * d6 - d5 * d4;
                        if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
                            const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
                            w[0] = 0; w[1] = 1 - t; w[2] = t;
                            q = b + t * (c - b);
                        } else {
                            const double den = 1.0 / ((va + vb) + vc);
                            const double v = vb * den, u = vc * den;
                            w[0] = 1.0 - v - u; w[1] = v; w[2] = u;
                            q = (a + v * ab) + u * ac;
                        }
                    }
                }
            }
        }
    }
    const V3 d = p - q;
    return dot(d, d);
}

struct Mesh {
    std::vector<V3> pts;
    const int32_t* faces;
    int n_faces;
};

// Uniform grid over the bounding box of a triangle mesh; each triangle is
// listed in every cell its bounding box overlaps.
struct Grid {
    V3 lo{}, cell{};
    int n = 1;
    std::vector<int> off, tri;
    const Mesh* mesh = nullptr;

    void build(const Mesh& m, int resolution) {
        mesh = &m;
        n = resolution;
        V3 hi{-1e300, -1e300, -1e300};
        lo = {1e300, 1e300, 1e300};
        for (const V3& p : m.pts) {
            lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
            hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
        }
        const double pad = 1e-9 + 1e-6 * std::max({hi.x - lo.x, hi.y - lo.y, hi.z - lo.z});
        lo = lo - V3{pad, pad, pad};
        hi = hi + V3{pad, pad, pad};
        cell = {(hi.x - lo.x) / n, (hi.y - lo.y) / n, (hi.z - lo.z) / n};
        std::vector<std::array<int, 6>> boxes(m.n_faces);
        std::vector<int> count(static_cast<size_t>(n) * n * n + 1, 0);
        for (int f = 0; f < m.n_faces; ++f) {
            V3 a = m.pts[m.faces[3 * f]], b = m.pts[m.faces[3 * f + 1]], c = m.pts[m.faces[3 * f + 2]];
            V3 mn{std::min({a.x, b.x, c.x}), std::min({a.y, b.y, c.y}), std::min({a.z, b.z, c.z})};
            V3 mx{std::max({a.x, b.x, c.x}), std::max({a.y, b.y, c.y}), std::max({a.z, b.z, c.z})};
            auto& bx = boxes[f];
            bx = {index(mn.x, lo.x, cell.x), index(mn.y, lo.y, cell.y), index(mn.z, lo.z, cell.z),
                  index(mx.x, lo.x, cell.x), index(mx.y, lo.y, cell.y), index(mx.z, lo.z, cell.z)};
            for (int z = bx[2]; z <= bx[5]; ++z)
                for (int y = bx[1]; y <= bx[4]; ++y)
                    for (int x = bx[0]; x <= bx[3]; ++x) count[id(x, y, z) + 1]++;
        }
        for (size_t i = 1; i < count.size(); ++i) count[i] += count[i - 1];
        off = count;
        tri.assign(static_cast<size_t>(off.back()), 0);
        std::vector<int> fill(off.begin(), off.end() - 1);
        for (int f = 0; f < m.n_faces; ++f) {
            const auto& bx = boxes[f];
            for (int z = bx[2]; z <= bx[5]; ++z)
                for (int y = bx[1]; y <= bx[4]; ++y)
                    for (int x = bx[0]; x <= bx[3]; ++x) tri[fill[id(x, y, z)]++] = f;
        }
    }
    int index(double v, double o, double c) const {
        int i = static_cast<int>(std::floor((v - o) / c));
        return std::min(std::max(i, 0), n - 1);
    }
    size_t id(int x, int y, int z) const { return (static_cast<size_t>(z) * n + y) * n + x; }

    // Exact closest triangle (lowest index on ties) and barycentric weights.
    int closest(V3 p, double w[3]) const {
        const int cx = index(p.x, lo.x, cell.x), cy = index(p.y, lo.y, cell.y), cz = index(p.z, lo.z, cell.z);
        double best = INFINITY;
        int best_f = -1;
        double bw[3] = {1, 0, 0};
        const double cmin = std::min({cell.x, cell.y, cell.z});
        for (int r = 0; r < n; ++r) {
            // cells at Chebyshev distance >= r from the query cell are at least (r - 1) * cmin away
            if (best_f >= 0) {
                const double reach = (r - 1) * cmin;
                if (reach > 0 && reach * reach > best) break;
            }
            for (int z = cz - r; z <= cz + r; ++z) {
                if (z < 0 || z >= n) continue;
                for (int y = cy - r; y <= cy + r; ++y) {
                    if (y < 0 || y >= n) continue;
                    for (int x = cx - r; x <= cx + r; ++x) {
                        if (x < 0 || x >= n) continue;
                        if (std::max({std::abs(x - cx), std::abs(y - cy), std::abs(z - cz)}) != r) continue;
                        const size_t c = id(x, y, z);
                        for (int k = off[c]; k < off[c + 1]; ++k) {
                            const int f = tri[k];
                            double ww[3];
                            const double d = closest_on_triangle(p, mesh->pts[mesh->faces[3 * f]],
                                                                 mesh->pts[mesh->faces[3 * f + 1]],
                                                                 mesh->pts[mesh->faces[3 * f + 2]], ww);
                            if (d < best || (d == best && f < best_f)) {
                                best = d;
                                best_f = f;
                                bw[0] = ww[0];
                                bw[1] = ww[1];
                                bw[2] = ww[2];
                            }
                        }
                    }
                }
            }
        }
        w[0] = bw[0];
        w[1] = bw[1];
        w[2] = bw[2];
        return best_f;
    }
};

template <typename F>
void parallel_for(int n, int threads, F fn) {
    threads = std::max(1, std::min(threads, n));
    std::vector<std::thread> pool;
    const int chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([=, &fn] {
            for (int i = t * chunk; i < std::min(n, (t + 1) * chunk); ++i) fn(i);
        });
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" int csg_stencil_build(const float* sphere, int n_sphere, const int32_t* sphere_faces, int n_sphere_faces,
                                 const double* resampling_points, int n_points, const int32_t* resampling_faces,
                                 int n_faces, int nx, int ny, int normalize, int threads, double* sphere_points_out,
                                 int32_t* surface_indices_out, double* surface_weights_out,
                                 int32_t* sheet_indices_out, double* sheet_weights_out, float* unit_points_out) {
    if (!sphere || n_sphere < 4 || !sphere_faces || n_sphere_faces < 4 || !resampling_points || n_points < 4 ||
        !resampling_faces || n_faces < 4 || nx < 1 || ny < 1 || !sphere_points_out || !surface_indices_out ||
        !surface_weights_out || !sheet_indices_out || !sheet_weights_out || !unit_points_out)
        return csg::fail(CSG_ERR_ARG, "stencil build: bad arguments");
    for (long long i = 0; i < 3LL * n_sphere_faces; ++i)
        if (sphere_faces[i] < 0 || sphere_faces[i] >= n_sphere)
            return csg::fail(CSG_ERR_TOPOLOGY, "stencil build: sphere face index out of range");
    for (long long i = 0; i < 3LL * n_faces; ++i)
        if (resampling_faces[i] < 0 || resampling_faces[i] >= n_points)
            return csg::fail(CSG_ERR_TOPOLOGY, "stencil build: resampling face index out of range");
    if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    // input sphere, optionally centred on its vertex mean and projected to unit length
    Mesh in{std::vector<V3>(n_sphere), sphere_faces, n_sphere_faces};
    V3 mean{0, 0, 0};
    for (int i = 0; i < n_sphere; ++i) {
        in.pts[i] = {sphere[3 * i], sphere[3 * i + 1], sphere[3 * i + 2]};
        mean = mean + in.pts[i];
    }
    mean = (1.0 / n_sphere) * mean;
    double radius = 0.0;
    for (int i = 0; i < n_sphere; ++i) {
        if (normalize) {
            V3 p = in.pts[i] - mean;
            const double len = std::sqrt(dot(p, p));
            if (!(len > 0.0)) return csg::fail(CSG_ERR_ARG, "stencil build: a sphere vertex sits at the centre");
            in.pts[i] = (1.0 / len) * p;
        }
        radius += std::sqrt(dot(in.pts[i], in.pts[i]));
    }
    radius = 0.975 * radius / n_sphere;
    const int res = std::max(8, std::min(128, static_cast<int>(std::cbrt(static_cast<double>(n_sphere_faces)) * 1.5)));
    Grid gin;
    gin.build(in, res);
    // sphere points: resampling-sphere directions moved onto the input sphere
    std::vector<V3> unit(n_points);
    for (int i = 0; i < n_points; ++i) {
        V3 p{resampling_points[3 * i], resampling_points[3 * i + 1], resampling_points[3 * i + 2]};
        unit[i] = (1.0 / std::sqrt(dot(p, p))) * p;
    }
    parallel_for(n_points, threads, [&](int i) {
        double w[3];
        const int f = gin.closest(unit[i], w);
        const int32_t* t = sphere_faces + 3 * f;
        const V3 q = (w[0] * in.pts[t[0]] + w[1] * in.pts[t[1]]) + w[2] * in.pts[t[2]];
        sphere_points_out[3 * i] = q.x;
        sphere_points_out[3 * i + 1] = q.y;
        sphere_points_out[3 * i + 2] = q.z;
        // surface barycentrics of the resampling point at 0.975 x the mean radius
        double w2[3];
        const int f2 = gin.closest(radius * unit[i], w2);
        for (int k = 0; k < 3; ++k) {
            surface_indices_out[3 * i + k] = sphere_faces[3 * f2 + k];
            surface_weights_out[3 * i + k] = w2[k];
        }
    });
    // sheet: cell centres on the unit-normalised sphere points
    Mesh us{std::vector<V3>(n_points), resampling_faces, n_faces};
    for (int i = 0; i < n_points; ++i) {
        V3 p{sphere_points_out[3 * i], sphere_points_out[3 * i + 1], sphere_points_out[3 * i + 2]};
        us.pts[i] = (1.0 / std::sqrt(dot(p, p))) * p;
    }
    Grid gus;
    gus.build(us, std::max(8, std::min(128, static_cast<int>(std::cbrt(static_cast<double>(n_faces)) * 1.5))));
    const double pi = 3.141592653589793;
    parallel_for(nx * ny, threads, [&](int cellid) {
        const int x = cellid % nx, y = cellid / nx;
        const double u = (x + 0.5) / nx, v = (y + 0.5) / ny;
        const V3 p{std::sin(v * pi) * std::cos(2.0 * pi * u), std::sin(v * pi) * std::sin(2.0 * pi * u),
                   std::cos(v * pi)};
        double w[3];
        const int f = gus.closest(p, w);
        for (int k = 0; k < 3; ++k) {
            sheet_indices_out[3 * cellid + k] = resampling_faces[3 * f + k];
            sheet_weights_out[3 * cellid + k] = w[k];
        }
    });
    for (int i = 0; i < n_sphere; ++i) {
        const V3 p = in.pts[i];
        const double len = std::sqrt(dot(p, p));
        unit_points_out[3 * i] = static_cast<float>(p.x / len);
        unit_points_out[3 * i + 1] = static_cast<float>(p.y / len);
        unit_points_out[3 * i + 2] = static_cast<float>(p.z / len);
    }
    return CSG_OK;
}
