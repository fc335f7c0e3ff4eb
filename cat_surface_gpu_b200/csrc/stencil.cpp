// Spherical resampling stencils (host C++, float64, deterministic, threaded).
//
// Builds the same stencil the reference's helper writes
// (native/cat_surface_stencil_builder.c:107-170, 355-464 in the reference
// project):
//   * the input sphere is centred on its vertex mean and unit-normalised
//     (unless `normalize` is 0); the resampling sphere's unit directions are
//     placed at centre + r u with centre = per-axis (min + max) of those
//     points and r = 0.975 x their mean length, as the helper places its
//     tetrahedral sphere (:406-421);
//   * surface barycentrics: for every placed resampling point, the input
//     triangle the helper's closest-polygon rule picks and the barycentric
//     weights of the picked point -- indices refer to the surface (same
//     topology as the sphere);
//   * sphere points: the input sphere interpolated with those weights (the
//     helper's resampled sphere, :424);
//   * sheet barycentrics: for every sheet cell centre (u, v) =
//     ((x + 0.5) / nx, (y + 0.5) / ny) mapped to the unit point
//     (sin(pi v) cos(2 pi u), sin(pi v) sin(2 pi u), cos(pi v)), the picked
//     triangle of the unit-normalised sphere points (:138-170);
//   * unit-sphere points of the input vertices.
// The resampling sphere (points + faces) is supplied by the caller.
//
// The closest-polygon rule is the one the reference restates for its
// rotation search (src/cat_surface_gpu/surface_rotation.py:354-425): project
// the query onto each triangle's plane; if the projection's parametric
// coordinates lie inside the triangle with a 1e-3 tolerance the candidate
// distance is the plane distance, otherwise it is the distance to the nearer
// of the two edges at the triangle's nearest vertex; the smallest candidate
// distance wins, ties to the lowest triangle index; the weights are those of
// the winning point (:335-352).  The search over a uniform grid of the
// triangles is exhaustive in effect: shells of cells are visited until no
// unvisited cell can hold a triangle whose candidate distance is smaller.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/catsurf_b200.h"
#include "errors.h"

namespace {

struct V3 {
    double x, y, z;
};
__host__ __device__ inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

__host__ __device__ inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Nearest point to p on segment [first, second] and its squared distance.
__host__ __device__ inline double segment_point(V3 p, V3 first, V3 second, V3& q) {
    const V3 dir = second - first, off = p - first;
    const double den = dot(dir, dir);
    double alpha = den != 0.0 ? dot(off, dir) / den : 0.0;
    alpha = alpha < 0.0 ? 0.0 : (alpha > 1.0 ? 1.0 : alpha);
    q = first + alpha * dir;
    const V3 d = p - q;
    return dot(d, d);
}

// Candidate distance of p to triangle abc under the closest-polygon rule
// (plane projection inside with a 1e-3 parametric tolerance, else the nearer
// edge at the nearest vertex) and the candidate point.  Shared by the host
// builder and the device kernels (one IEEE rounding per operation on both:
// no contraction on either side).
__host__ __device__ double locate_on_triangle(V3 p, V3 a, V3 b, V3 c, V3& point) {
    const V3 ea = b - a, eb = c - a;
    const V3 n = cross(ea, eb);
    const double nsq = dot(n, n);
    const double t = nsq != 0.0 ? dot(a - p, n) / nsq : 0.0;
    const V3 proj = p + t * n;
    const V3 po = proj - a;
    const double xx = dot(ea, ea), xy = dot(ea, eb), xv = dot(ea, po), yy = dot(eb, eb), yv = dot(eb, po);
    const double den = xx * yy - xy * xy;
    const double xpos = den != 0.0 ? (xv * yy - yv * xy) / den : 0.0;
    const double ypos = den != 0.0 ? (yv * xx - xv * xy) / den : 0.0;
    const double tol = 1.0e-3, top = 1.0 + tol;
    const double sum = xpos + ypos;
    if (den != 0.0 && xpos >= -tol && xpos <= top && ypos >= -tol && ypos <= top && sum >= -tol && sum <= top) {
        point = proj;
        return t * t * nsq;
    }
    const V3 v[3] = {a, b, c};
    double vd[3];
    for (int k = 0; k < 3; ++k) {
        const V3 d = p - v[k];
        vd[k] = dot(d, d);
    }
    int cv = 0;
    if (vd[1] < vd[cv]) cv = 1;
    if (vd[2] < vd[cv]) cv = 2;
    V3 q1, q2;
    const double d1 = segment_point(p, v[(cv + 2) % 3], v[cv], q1);
    const double d2 = segment_point(p, v[cv], v[(cv + 1) % 3], q2);
    if (d1 < d2) {
        point = q1;
        return d1;
    }
    point = q2;
    return d2;
}

// Barycentric weights of p in triangle abc: for each vertex, the offset of
// p from the opposite edge along the in-plane normal of that edge, over the
// vertex's own offset (the reference's three-cross-product form).
__host__ __device__ void point_weights(V3 p, V3 a, V3 b, V3 c, double w[3]) {
    const V3 t[3] = {a, b, c};
    for (int k = 0; k < 3; ++k) {
        const V3 first = t[(k + 1) % 3], second = t[(k + 2) % 3], third = t[k];
        const V3 po = p - first, hz = second - first, up = third - first;
        const V3 vert = cross(cross(hz, up), hz);
        w[k] = dot(po, vert) / dot(up, vert);
    }
}

// Upper bound on how far a point the rule accepts as inside (within the
// tolerance) can lie from its triangle: 3e-3 of the longest edge, doubled.
double tolerance_reach(const std::vector<V3>& pts, const int32_t* faces, int n_faces) {
    double longest = 0.0;
    for (int f = 0; f < n_faces; ++f)
        for (int k = 0; k < 3; ++k) {
            const V3 d = pts[faces[3 * f + k]] - pts[faces[3 * f + (k + 1) % 3]];
            longest = std::max(longest, std::sqrt(dot(d, d)));
        }
    return 6.0e-3 * longest;
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
    double slack = 0.0;  // tolerance_reach of the mesh
    std::vector<int> off, tri;
    const Mesh* mesh = nullptr;

    void build(const Mesh& m, int resolution) {
        mesh = &m;
        n = resolution;
        slack = tolerance_reach(m.pts, m.faces, m.n_faces);
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

    // The triangle the closest-polygon rule picks (lowest index on ties) and
    // the weights of its candidate point.  A triangle in a cell at Chebyshev
    // distance >= r lies at least (r - 1) * cmin away, so its candidate
    // distance is at least ((r - 1) * cmin - slack)^2.
    int locate(V3 p, double w[3]) const {
        const int cx = index(p.x, lo.x, cell.x), cy = index(p.y, lo.y, cell.y), cz = index(p.z, lo.z, cell.z);
        double best = INFINITY;
        int best_f = -1;
        V3 bq{0, 0, 0};
        const double cmin = std::min({cell.x, cell.y, cell.z});
        for (int r = 0; r < n; ++r) {
            if (best_f >= 0) {
                const double reach = (r - 1) * cmin - slack;
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
                            V3 q;
                            const double d = locate_on_triangle(p, mesh->pts[mesh->faces[3 * f]],
                                                                mesh->pts[mesh->faces[3 * f + 1]],
                                                                mesh->pts[mesh->faces[3 * f + 2]], q);
                            if (d < best || (d == best && f < best_f)) {
                                best = d;
                                best_f = f;
                                bq = q;
                            }
                        }
                    }
                }
            }
        }
        if (best_f >= 0)
            point_weights(bq, mesh->pts[mesh->faces[3 * best_f]], mesh->pts[mesh->faces[3 * best_f + 1]],
                          mesh->pts[mesh->faces[3 * best_f + 2]], w);
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

int grid_resolution(int n_faces) {
    return std::max(8, std::min(128, static_cast<int>(std::cbrt(static_cast<double>(n_faces)) * 1.5)));
}

// Host preparation shared by both builders: argument checks, the input
// sphere (optionally centred and unit-normalised), 0.975 x its mean radius,
// the unit resampling directions and the sheet cell-centre points.
struct Prepared {
    std::vector<V3> pts;
    double radius = 0.0;
    V3 centre{0, 0, 0};       // per-axis (min + max) of pts: where the resampling sphere is placed
    std::vector<V3> unit;
    std::vector<V3> placed;   // centre + radius * unit
    std::shared_ptr<const std::vector<V3>> sheet;  // shared by every build of one sheet size
};

// Unit directions of the nx x ny sheet cell centres (latitude v, longitude u).
// They depend on the sheet size alone, so one table per size is kept for the
// life of the process; builds running in parallel threads share it.
std::shared_ptr<const std::vector<V3>> sheet_directions(int nx, int ny) {
    static std::mutex lock;
    static std::map<std::pair<int, int>, std::shared_ptr<const std::vector<V3>>> tables;
    std::lock_guard<std::mutex> guard(lock);
    auto& slot = tables[{nx, ny}];
    if (!slot) {
        const double pi = 3.141592653589793;
        auto table = std::make_shared<std::vector<V3>>(static_cast<size_t>(nx) * ny);
        for (int cellid = 0; cellid < nx * ny; ++cellid) {
            const int x = cellid % nx, y = cellid / nx;
            const double u = (x + 0.5) / nx, v = (y + 0.5) / ny;
            (*table)[cellid] = {std::sin(v * pi) * std::cos(2.0 * pi * u), std::sin(v * pi) * std::sin(2.0 * pi * u),
                                std::cos(v * pi)};
        }
        slot = std::move(table);
    }
    return slot;
}

int prepare(const float* sphere, int n_sphere, const int32_t* sphere_faces, int n_sphere_faces,
            const double* resampling_points, int n_points, const int32_t* resampling_faces, int n_faces, int nx, int ny,
            int normalize, Prepared& out) {
    if (!sphere || n_sphere < 4 || !sphere_faces || n_sphere_faces < 4 || !resampling_points || n_points < 4 ||
        !resampling_faces || n_faces < 4 || nx < 1 || ny < 1)
        return csg::fail(CSG_ERR_ARG, "stencil build: bad arguments");
    for (long long i = 0; i < 3LL * n_sphere_faces; ++i)
        if (sphere_faces[i] < 0 || sphere_faces[i] >= n_sphere)
            return csg::fail(CSG_ERR_TOPOLOGY, "stencil build: sphere face index out of range");
    for (long long i = 0; i < 3LL * n_faces; ++i)
        if (resampling_faces[i] < 0 || resampling_faces[i] >= n_points)
            return csg::fail(CSG_ERR_TOPOLOGY, "stencil build: resampling face index out of range");
    out.pts.assign(n_sphere, V3{0, 0, 0});
    V3 mean{0, 0, 0};
    for (int i = 0; i < n_sphere; ++i) {
        out.pts[i] = {sphere[3 * i], sphere[3 * i + 1], sphere[3 * i + 2]};
        mean = mean + out.pts[i];
    }
    mean = (1.0 / n_sphere) * mean;
    double radius = 0.0;
    for (int i = 0; i < n_sphere; ++i) {
        if (normalize) {
            V3 p = out.pts[i] - mean;
            const double len = std::sqrt(dot(p, p));
            if (!(len > 0.0)) return csg::fail(CSG_ERR_ARG, "stencil build: a sphere vertex sits at the centre");
            out.pts[i] = (1.0 / len) * p;
        }
        radius += std::sqrt(dot(out.pts[i], out.pts[i]));
    }
    out.radius = 0.975 * radius / n_sphere;
    V3 lo = out.pts[0], hi = out.pts[0];
    for (const V3& p : out.pts) {
        lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
        hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
    }
    out.centre = lo + hi;
    out.unit.assign(n_points, V3{0, 0, 0});
    out.placed.assign(n_points, V3{0, 0, 0});
    for (int i = 0; i < n_points; ++i) {
        V3 p{resampling_points[3 * i], resampling_points[3 * i + 1], resampling_points[3 * i + 2]};
        out.unit[i] = (1.0 / std::sqrt(dot(p, p))) * p;
        out.placed[i] = out.centre + out.radius * out.unit[i];
    }
    out.sheet = sheet_directions(nx, ny);
    return CSG_OK;
}

void write_unit_points(const Prepared& prep, float* unit_points_out) {
    for (size_t i = 0; i < prep.pts.size(); ++i) {
        const V3 p = prep.pts[i];
        const double len = std::sqrt(dot(p, p));
        unit_points_out[3 * i] = static_cast<float>(p.x / len);
        unit_points_out[3 * i + 1] = static_cast<float>(p.y / len);
        unit_points_out[3 * i + 2] = static_cast<float>(p.z / len);
    }
}

// ------------------------------------------------------------ device builder
//
// The same closest-polygon queries on the GPU: one thread per query, the
// host's shell search over a uniform grid (built on the device: bounding box
// by min/max reduction, per-cell counts by atomics, a two-level scan, and an
// atomic fill whose in-cell order does not matter because the search visits
// every triangle that can win and breaks ties by the lowest triangle index).
// Results are bit-identical to the host builder.

constexpr int kScanBlock = 1024;

struct GridParams {
    double lo[3];
    double cell[3];
    double cmin;
    double slack;  // an upper bound on the mesh's tolerance_reach
};

__device__ __forceinline__ int cell_index(double v, double o, double c, int n) {
    const int i = static_cast<int>(floor((v - o) / c));
    return min(max(i, 0), n - 1);
}

__device__ __forceinline__ V3 load_point(const double* pts, int i) {
    return {__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2)};
}

// Bounding box of the points padded like Grid::build, then the cell sizes.
__global__ void k_grid_box(const double* __restrict__ pts, int n_pts, int res, double slack,
                           GridParams* __restrict__ gp) {
    __shared__ double lo_s[3][kScanBlock], hi_s[3][kScanBlock];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = threadIdx.x; i < n_pts; i += blockDim.x)
        for (int k = 0; k < 3; ++k) {
            const double v = pts[3 * i + k];
            lo[k] = fmin(lo[k], v);
            hi[k] = fmax(hi[k], v);
        }
    for (int k = 0; k < 3; ++k) {
        lo_s[k][threadIdx.x] = lo[k];
        hi_s[k][threadIdx.x] = hi[k];
    }
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride)
            for (int k = 0; k < 3; ++k) {
                lo_s[k][threadIdx.x] = fmin(lo_s[k][threadIdx.x], lo_s[k][threadIdx.x + stride]);
                hi_s[k][threadIdx.x] = fmax(hi_s[k][threadIdx.x], hi_s[k][threadIdx.x + stride]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double ext = fmax(fmax(hi_s[0][0] - lo_s[0][0], hi_s[1][0] - lo_s[1][0]), hi_s[2][0] - lo_s[2][0]);
        const double pad = 1e-9 + 1e-6 * ext;
        for (int k = 0; k < 3; ++k) {
            gp->lo[k] = lo_s[k][0] - pad;
            gp->cell[k] = ((hi_s[k][0] + pad) - gp->lo[k]) / res;
        }
        gp->cmin = fmin(fmin(gp->cell[0], gp->cell[1]), gp->cell[2]);
        gp->slack = slack;
    }
}

__device__ __forceinline__ void face_box(const double* pts, const int* faces, int f, const GridParams& g, int res,
                                         int b[6]) {
    const V3 a = load_point(pts, faces[3 * f]), bb = load_point(pts, faces[3 * f + 1]),
             c = load_point(pts, faces[3 * f + 2]);
    const double mn[3] = {fmin(fmin(a.x, bb.x), c.x), fmin(fmin(a.y, bb.y), c.y), fmin(fmin(a.z, bb.z), c.z)};
    const double mx[3] = {fmax(fmax(a.x, bb.x), c.x), fmax(fmax(a.y, bb.y), c.y), fmax(fmax(a.z, bb.z), c.z)};
    for (int k = 0; k < 3; ++k) {
        b[k] = cell_index(mn[k], g.lo[k], g.cell[k], res);
        b[3 + k] = cell_index(mx[k], g.lo[k], g.cell[k], res);
    }
}

__global__ void k_grid_count(const double* __restrict__ pts, const int* __restrict__ faces, int n_faces,
                             const GridParams* __restrict__ gp, int res, int* __restrict__ counts) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const GridParams g = *gp;
    int b[6];
    face_box(pts, faces, f, g, res, b);
    for (int z = b[2]; z <= b[5]; ++z)
        for (int y = b[1]; y <= b[4]; ++y)
            for (int x = b[0]; x <= b[3]; ++x)
                atomicAdd(counts + (static_cast<size_t>(z) * res + y) * res + x + 1, 1);
}

// Inclusive scan of `data` in blocks of kScanBlock (block totals to `sums`).
__global__ void k_scan_block(int* __restrict__ data, int n, int* __restrict__ sums) {
    __shared__ int buf[kScanBlock];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    buf[threadIdx.x] = i < n ? data[i] : 0;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
        const int v = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
        __syncthreads();
        buf[threadIdx.x] += v;
        __syncthreads();
    }
    if (i < n) data[i] = buf[threadIdx.x];
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = buf[threadIdx.x];
}

// Exclusive scan of the block totals by one block, in place.
__global__ void k_scan_sums(int* __restrict__ sums, int nblocks) {
    __shared__ int buf[kScanBlock];
    int carry = 0;
    for (int base = 0; base < nblocks; base += kScanBlock) {
        const int i = base + threadIdx.x;
        const int own = i < nblocks ? sums[i] : 0;
        buf[threadIdx.x] = own;
        __syncthreads();
        for (int off = 1; off < kScanBlock; off <<= 1) {
            const int v = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += v;
            __syncthreads();
        }
        if (i < nblocks) sums[i] = carry + buf[threadIdx.x] - own;
        const int total = buf[kScanBlock - 1];
        __syncthreads();
        carry += total;
    }
}

__global__ void k_scan_add(int* __restrict__ data, int n, const int* __restrict__ sums, int* __restrict__ cursor) {
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i >= n) return;
    const int v = data[i] + sums[blockIdx.x];
    data[i] = v;
    if (cursor && i + 1 < n) cursor[i] = v;  // fill cursor of cell i starts at offset i
}

__global__ void k_grid_fill(const double* __restrict__ pts, const int* __restrict__ faces, int n_faces,
                            const GridParams* __restrict__ gp, int res, const int* __restrict__ offsets,
                            int* __restrict__ cursor, int* __restrict__ tri, long long capacity,
                            int* __restrict__ overflow) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const long long total = offsets[static_cast<size_t>(res) * res * res];
    if (total > capacity) {
        if (f == 0) atomicExch(overflow, 1);
        return;
    }
    const GridParams g = *gp;
    int b[6];
    face_box(pts, faces, f, g, res, b);
    for (int z = b[2]; z <= b[5]; ++z)
        for (int y = b[1]; y <= b[4]; ++y)
            for (int x = b[0]; x <= b[3]; ++x)
                tri[atomicAdd(cursor + (static_cast<size_t>(z) * res + y) * res + x, 1)] = f;
}

struct DevMesh {
    const double* pts;
    const int* faces;
    const int* off;
    const int* tri;
    const GridParams* gp;
    int res;
};

// Grid::locate on the device by a group of G lanes: the triangle the
// closest-polygon rule picks (lowest index on ties) and the weights of its
// candidate point.  The lanes split each shell's cells, keep their own
// lexicographic (distance, face) minimum, and the group takes the minimum of
// those after the shell.  The pick is the minimum over the same candidate set
// as a one-lane scan (the same shells, the same stop test on the same running
// minimum), so the face, its candidate point and weights are the same.
template <int G>
__device__ int locate_group(const DevMesh& m, V3 p, double w[3]) {
    const int lane = threadIdx.x & 31, glane = lane & (G - 1), gbase = lane & ~(G - 1);
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << gbase;
    const GridParams g = *m.gp;
    const int n = m.res;
    const int cx = cell_index(p.x, g.lo[0], g.cell[0], n), cy = cell_index(p.y, g.lo[1], g.cell[1], n),
              cz = cell_index(p.z, g.lo[2], g.cell[2], n);
    double best = INFINITY;
    int best_f = -1;
    V3 bq{0, 0, 0};
    for (int r = 0; r < n; ++r) {
        if (best_f >= 0) {
            const double reach = (r - 1) * g.cmin - g.slack;
            if (reach > 0 && reach * reach > best) break;
        }
        const int side = 2 * r + 1, plane = side * side;
        for (int idx = glane; idx < plane * side; idx += G) {
            const int dz = idx / plane, rem = idx - dz * plane, dy = rem / side, dx = rem - dy * side;
            const int z = cz - r + dz, y = cy - r + dy, x = cx - r + dx;
            if (z < 0 || z >= n || y < 0 || y >= n || x < 0 || x >= n) continue;
            if (max(max(abs(x - cx), abs(y - cy)), abs(z - cz)) != r) continue;
            const size_t c = (static_cast<size_t>(z) * n + y) * n + x;
            const int k1 = __ldg(m.off + c + 1);
            for (int k = __ldg(m.off + c); k < k1; ++k) {
                const int f = __ldg(m.tri + k);
                V3 q;
                const double d = locate_on_triangle(p, load_point(m.pts, __ldg(m.faces + 3 * f)),
                                                    load_point(m.pts, __ldg(m.faces + 3 * f + 1)),
                                                    load_point(m.pts, __ldg(m.faces + 3 * f + 2)), q);
                if (d < best || (d == best && f < best_f)) {
                    best = d;
                    best_f = f;
                    bq = q;
                }
            }
        }
        double gd = best;
        int gf = best_f;
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) {
            const double od = __shfl_xor_sync(gmask, gd, off);
            const int of = __shfl_xor_sync(gmask, gf, off);
            if (od < gd || (od == gd && of < gf)) {
                gd = od;
                gf = of;
            }
        }
        const unsigned owners = __ballot_sync(gmask, best == gd && best_f == gf) & gmask;
        const int src = __ffs(owners) - 1;
        bq.x = __shfl_sync(gmask, bq.x, src);
        bq.y = __shfl_sync(gmask, bq.y, src);
        bq.z = __shfl_sync(gmask, bq.z, src);
        best = gd;
        best_f = gf;
    }
    if (best_f >= 0)
        point_weights(bq, load_point(m.pts, __ldg(m.faces + 3 * best_f)),
                      load_point(m.pts, __ldg(m.faces + 3 * best_f + 1)),
                      load_point(m.pts, __ldg(m.faces + 3 * best_f + 2)), w);
    return best_f;
}

constexpr int kLocateLanes = 4;  // measured: 4 lanes per query beat 1 and 8 on 61k-vertex spheres

// flag: 1 = a grid overflowed its capacity, 2 = a query found no triangle
// (non-finite input); later kernels skip their work once it is set.
__global__ void k_stencil_points(DevMesh in, const double* __restrict__ placed, int n_points, int* __restrict__ flag,
                                 double* __restrict__ sphere_points, double* __restrict__ unit_sphere,
                                 int* __restrict__ sidx, double* __restrict__ sw) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) / kLocateLanes;
    if (i >= n_points) return;  // the whole group
    const int gbase = (threadIdx.x & 31) & ~(kLocateLanes - 1);
    const unsigned gmask = (kLocateLanes == 32 ? 0xffffffffu : ((1u << kLocateLanes) - 1u)) << gbase;
    if (__shfl_sync(gmask, *flag, gbase)) return;  // one reading per group
    double w[3];
    const int f = locate_group<kLocateLanes>(in, load_point(placed, i), w);
    if ((threadIdx.x & (kLocateLanes - 1)) != 0) return;
    if (f < 0) {
        atomicExch(flag, 2);
        return;
    }
    const int* t = in.faces + 3 * f;
    const V3 q = (w[0] * load_point(in.pts, t[0]) + w[1] * load_point(in.pts, t[1])) + w[2] * load_point(in.pts, t[2]);
    sphere_points[3 * i] = q.x;
    sphere_points[3 * i + 1] = q.y;
    sphere_points[3 * i + 2] = q.z;
    const V3 un = (1.0 / sqrt(dot(q, q))) * q;
    unit_sphere[3 * i] = un.x;
    unit_sphere[3 * i + 1] = un.y;
    unit_sphere[3 * i + 2] = un.z;
    for (int k = 0; k < 3; ++k) {
        sidx[3 * i + k] = t[k];
        sw[3 * i + k] = w[k];
    }
}

__global__ void k_stencil_sheet(DevMesh us, const double* __restrict__ sheet, int n_cells, int* __restrict__ flag,
                                int* __restrict__ idx, double* __restrict__ wts) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) / kLocateLanes;
    if (i >= n_cells) return;  // the whole group
    const int gbase = (threadIdx.x & 31) & ~(kLocateLanes - 1);
    const unsigned gmask = (kLocateLanes == 32 ? 0xffffffffu : ((1u << kLocateLanes) - 1u)) << gbase;
    if (__shfl_sync(gmask, *flag, gbase)) return;  // one reading per group
    double w[3];
    const int f = locate_group<kLocateLanes>(us, load_point(sheet, i), w);
    if ((threadIdx.x & (kLocateLanes - 1)) != 0) return;
    if (f < 0) {
        atomicExch(flag, 2);
        return;
    }
    for (int k = 0; k < 3; ++k) {
        idx[3 * i + k] = us.faces[3 * f + k];
        wts[3 * i + k] = w[k];
    }
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct DeviceLayout {
    size_t in_pts, in_faces, unit, r_faces, sheet, sp, us, sidx, sw, shidx, shw;
    size_t gp_a, gp_b, flag, sums;
    size_t off_a, cur_a, tri_a, off_b, cur_b, tri_b;
    size_t total;
    long long cap_a, cap_b;
};

DeviceLayout layout(int n_sphere, int n_sphere_faces, int n_points, int n_faces, int nx, int ny) {
    DeviceLayout L{};
    const int res_a = grid_resolution(n_sphere_faces), res_b = grid_resolution(n_faces);
    const size_t cells_a = static_cast<size_t>(res_a) * res_a * res_a, cells_b = static_cast<size_t>(res_b) * res_b * res_b;
    const size_t cells = static_cast<size_t>(nx) * ny;
    L.cap_a = 16LL * n_sphere_faces + 4096;
    L.cap_b = 16LL * n_faces + 4096;
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t here = at;
        at += align256(bytes);
        return here;
    };
    L.in_pts = take(24ULL * n_sphere);
    L.in_faces = take(12ULL * n_sphere_faces);
    L.unit = take(24ULL * n_points);
    L.r_faces = take(12ULL * n_faces);
    L.sheet = take(24ULL * cells);
    L.sp = take(24ULL * n_points);
    L.us = take(24ULL * n_points);
    L.sidx = take(12ULL * n_points);
    L.sw = take(24ULL * n_points);
    L.shidx = take(12ULL * cells);
    L.shw = take(24ULL * cells);
    L.gp_a = take(sizeof(GridParams));
    L.gp_b = take(sizeof(GridParams));
    L.flag = take(sizeof(int));
    L.sums = take(sizeof(int) * ((std::max(cells_a, cells_b) + 1) / kScanBlock + 2));
    L.off_a = take(4ULL * (cells_a + 1));
    L.cur_a = take(4ULL * cells_a);
    L.tri_a = take(4ULL * static_cast<size_t>(L.cap_a));
    L.off_b = take(4ULL * (cells_b + 1));
    L.cur_b = take(4ULL * cells_b);
    L.tri_b = take(4ULL * static_cast<size_t>(L.cap_b));
    L.total = at;
    return L;
}

int build_grid_device(char* base, const double* pts, int n_pts, const int* faces, int n_faces, int res,
                      double slack, size_t gp_at, size_t off_at, size_t cur_at, size_t tri_at, long long cap,
                      size_t sums_at, size_t flag_at, cudaStream_t s) {
    const size_t cells = static_cast<size_t>(res) * res * res;
    GridParams* gp = reinterpret_cast<GridParams*>(base + gp_at);
    int* off = reinterpret_cast<int*>(base + off_at);
    int* cur = reinterpret_cast<int*>(base + cur_at);
    int* sums = reinterpret_cast<int*>(base + sums_at);
    (csg::note_launch(), k_grid_box<<<1, kScanBlock, 0, s>>>(pts, n_pts, res, slack, gp));
    CSG_CUDA_CHECK(cudaMemsetAsync(off, 0, 4 * (cells + 1), s));
    const unsigned fb = static_cast<unsigned>((n_faces + 255) / 256);
    (csg::note_launch(), k_grid_count<<<fb, 256, 0, s>>>(pts, faces, n_faces, gp, res, off));
    const int n = static_cast<int>(cells + 1);
    const int nblocks = (n + kScanBlock - 1) / kScanBlock;
    (csg::note_launch(), k_scan_block<<<nblocks, kScanBlock, 0, s>>>(off, n, sums));
    (csg::note_launch(), k_scan_sums<<<1, kScanBlock, 0, s>>>(sums, nblocks));
    (csg::note_launch(), k_scan_add<<<nblocks, kScanBlock, 0, s>>>(off, n, sums, cur));
    (csg::note_launch(), k_grid_fill<<<fb, 256, 0, s>>>(pts, faces, n_faces, gp, res, off, cur,
                                                        reinterpret_cast<int*>(base + tri_at), cap,
                                                        reinterpret_cast<int*>(base + flag_at)));
    return CSG_OK;
}

}  // namespace

extern "C" int csg_stencil_build(const float* sphere, int n_sphere, const int32_t* sphere_faces, int n_sphere_faces,
                                 const double* resampling_points, int n_points, const int32_t* resampling_faces,
                                 int n_faces, int nx, int ny, int normalize, int threads, double* sphere_points_out,
                                 int32_t* surface_indices_out, double* surface_weights_out,
                                 int32_t* sheet_indices_out, double* sheet_weights_out, float* unit_points_out) {
    if (!sphere_points_out || !surface_indices_out || !surface_weights_out || !sheet_indices_out ||
        !sheet_weights_out || !unit_points_out)
        return csg::fail(CSG_ERR_ARG, "stencil build: bad arguments");
    Prepared prep;
    int rc = prepare(sphere, n_sphere, sphere_faces, n_sphere_faces, resampling_points, n_points, resampling_faces,
                     n_faces, nx, ny, normalize, prep);
    if (rc) return rc;
    if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    std::atomic<int> failed{0};
    Mesh in{prep.pts, sphere_faces, n_sphere_faces};
    Grid gin;
    gin.build(in, grid_resolution(n_sphere_faces));
    // surface barycentrics of each placed resampling point, and the input sphere interpolated there
    parallel_for(n_points, threads, [&](int i) {
        double w[3];
        const int f = gin.locate(prep.placed[i], w);
        if (f < 0) {
            failed = 1;
            return;
        }
        const int32_t* t = sphere_faces + 3 * f;
        const V3 q = (w[0] * in.pts[t[0]] + w[1] * in.pts[t[1]]) + w[2] * in.pts[t[2]];
        sphere_points_out[3 * i] = q.x;
        sphere_points_out[3 * i + 1] = q.y;
        sphere_points_out[3 * i + 2] = q.z;
        for (int k = 0; k < 3; ++k) {
            surface_indices_out[3 * i + k] = t[k];
            surface_weights_out[3 * i + k] = w[k];
        }
    });
    // sheet: cell centres on the unit-normalised sphere points
    if (failed) return csg::fail(CSG_ERR_ARG, "stencil build: a query found no triangle (non-finite input)");
    Mesh us{std::vector<V3>(n_points), resampling_faces, n_faces};
    for (int i = 0; i < n_points; ++i) {
        V3 p{sphere_points_out[3 * i], sphere_points_out[3 * i + 1], sphere_points_out[3 * i + 2]};
        us.pts[i] = (1.0 / std::sqrt(dot(p, p))) * p;
    }
    Grid gus;
    gus.build(us, grid_resolution(n_faces));
    parallel_for(nx * ny, threads, [&](int cellid) {
        double w[3];
        const int f = gus.locate((*prep.sheet)[cellid], w);
        if (f < 0) {
            failed = 1;
            return;
        }
        for (int k = 0; k < 3; ++k) {
            sheet_indices_out[3 * cellid + k] = resampling_faces[3 * f + k];
            sheet_weights_out[3 * cellid + k] = w[k];
        }
    });
    if (failed) return csg::fail(CSG_ERR_ARG, "stencil build: a query found no triangle (non-finite input)");
    write_unit_points(prep, unit_points_out);
    return CSG_OK;
}

extern "C" size_t csg_stencil_scratch_bytes(int n_sphere, int n_sphere_faces, int n_points, int n_faces, int nx,
                                            int ny) {
    if (n_sphere < 4 || n_sphere_faces < 4 || n_points < 4 || n_faces < 4 || nx < 1 || ny < 1) return 0;
    return layout(n_sphere, n_sphere_faces, n_points, n_faces, nx, ny).total;
}

extern "C" int csg_stencil_build_device(const float* sphere, int n_sphere, const int32_t* sphere_faces,
                                        int n_sphere_faces, const double* resampling_points, int n_points,
                                        const int32_t* resampling_faces, int n_faces, int nx, int ny, int normalize,
                                        double* sphere_points_out, int32_t* surface_indices_out,
                                        double* surface_weights_out, int32_t* sheet_indices_out,
                                        double* sheet_weights_out, float* unit_points_out, void* scratch,
                                        size_t scratch_bytes, csg_stream_t stream) {
    if (!sphere_points_out || !surface_indices_out || !surface_weights_out || !sheet_indices_out ||
        !sheet_weights_out || !unit_points_out || !scratch)
        return csg::fail(CSG_ERR_ARG, "stencil build (device): bad arguments");
    Prepared prep;
    int rc = prepare(sphere, n_sphere, sphere_faces, n_sphere_faces, resampling_points, n_points, resampling_faces,
                     n_faces, nx, ny, normalize, prep);
    if (rc) return rc;
    const DeviceLayout L = layout(n_sphere, n_sphere_faces, n_points, n_faces, nx, ny);
    if (scratch_bytes < L.total) return csg::fail(CSG_ERR_ARG, "stencil build (device): scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(scratch);
    const int cells = nx * ny;
    CSG_CUDA_CHECK(cudaMemcpyAsync(base + L.in_pts, prep.pts.data(), 24ULL * n_sphere, cudaMemcpyHostToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(base + L.in_faces, sphere_faces, 12ULL * n_sphere_faces, cudaMemcpyHostToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(base + L.unit, prep.placed.data(), 24ULL * n_points, cudaMemcpyHostToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(base + L.r_faces, resampling_faces, 12ULL * n_faces, cudaMemcpyHostToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(base + L.sheet, prep.sheet->data(), 24ULL * cells, cudaMemcpyHostToDevice, s));
    CSG_CUDA_CHECK(cudaMemsetAsync(base + L.flag, 0, sizeof(int), s));
    const int res_a = grid_resolution(n_sphere_faces), res_b = grid_resolution(n_faces);
    const double* in_pts = reinterpret_cast<const double*>(base + L.in_pts);
    const int* in_faces = reinterpret_cast<const int*>(base + L.in_faces);
    const int* r_faces = reinterpret_cast<const int*>(base + L.r_faces);
    int* flag = reinterpret_cast<int*>(base + L.flag);
    // the sheet mesh (the unit-normalised sphere points) is built on the device: bound its tolerance
    // reach by four times that of the unit resampling directions it stays close to
    rc = build_grid_device(base, in_pts, n_sphere, in_faces, n_sphere_faces, res_a,
                           tolerance_reach(prep.pts, sphere_faces, n_sphere_faces), L.gp_a, L.off_a, L.cur_a, L.tri_a,
                           L.cap_a, L.sums, L.flag, s);
    if (rc) return rc;
    DevMesh in{in_pts, in_faces, reinterpret_cast<const int*>(base + L.off_a),
               reinterpret_cast<const int*>(base + L.tri_a), reinterpret_cast<const GridParams*>(base + L.gp_a), res_a};
    double* sp = reinterpret_cast<double*>(base + L.sp);
    double* us = reinterpret_cast<double*>(base + L.us);
    CSG_CUDA_CHECK(cudaMemsetAsync(us, 0, 24ULL * n_points, s));
    (csg::note_launch(), k_stencil_points<<<(n_points * kLocateLanes + 127) / 128, 128, 0, s>>>(
        in, reinterpret_cast<const double*>(base + L.unit), n_points, flag, sp, us,
        reinterpret_cast<int*>(base + L.sidx), reinterpret_cast<double*>(base + L.sw)));
    rc = build_grid_device(base, us, n_points, r_faces, n_faces, res_b,
                           4.0 * tolerance_reach(prep.unit, resampling_faces, n_faces), L.gp_b, L.off_b, L.cur_b,
                           L.tri_b, L.cap_b, L.sums, L.flag, s);
    if (rc) return rc;
    DevMesh um{us, r_faces, reinterpret_cast<const int*>(base + L.off_b), reinterpret_cast<const int*>(base + L.tri_b),
               reinterpret_cast<const GridParams*>(base + L.gp_b), res_b};
    (csg::note_launch(), k_stencil_sheet<<<(cells * kLocateLanes + 127) / 128, 128, 0, s>>>(
        um, reinterpret_cast<const double*>(base + L.sheet), cells, flag, reinterpret_cast<int*>(base + L.shidx),
        reinterpret_cast<double*>(base + L.shw)));
    CSG_CUDA_CHECK(cudaGetLastError());
    int overflow = 0;
    CSG_CUDA_CHECK(cudaMemcpyAsync(&overflow, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(sphere_points_out, sp, 24ULL * n_points, cudaMemcpyDeviceToHost, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(surface_indices_out, base + L.sidx, 12ULL * n_points, cudaMemcpyDeviceToHost, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(surface_weights_out, base + L.sw, 24ULL * n_points, cudaMemcpyDeviceToHost, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(sheet_indices_out, base + L.shidx, 12ULL * cells, cudaMemcpyDeviceToHost, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(sheet_weights_out, base + L.shw, 24ULL * cells, cudaMemcpyDeviceToHost, s));
    write_unit_points(prep, unit_points_out);
    CSG_CUDA_CHECK(cudaStreamSynchronize(s));
    if (overflow == 1)
        return csg::fail(CSG_ERR_UNSUPPORTED, "stencil build (device): a grid cell list exceeded its capacity "
                                              "(triangles far larger than the grid cells); use the host builder");
    if (overflow)
        return csg::fail(CSG_ERR_ARG, "stencil build (device): a query found no triangle (non-finite input)");
    return CSG_OK;
}
