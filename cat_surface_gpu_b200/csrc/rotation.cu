// SurfWarp initial-rotation search on sm_100a: closest-triangle location of
// rotated source points on the target sphere and the SSD of the resampled
// target feature, for many candidate rotations and many surfaces at once.
//
// Follows src/cat_surface_gpu/surface_rotation.py: grid index (58-120),
// candidate query (455-477), closest point per candidate triangle -- plane
// projection with a 1e-3 inside tolerance, else the nearer of the two edges at
// the nearest vertex -- and the first minimum over candidates (354-453),
// barycentric weights (335-352) and the float64 SSD (512-546).  Geometry is
// float32 with one rounding per operation (compiled with --fmad=false):
// 3-term dot products are (a0 b0 + a1 b1) + a2 b2.
//
// Work decomposition: one work item = (surface, candidate, tile of kTile
// source points).  A persistent grid walks the flattened item list, so any
// mix of surfaces of uneven size and candidate counts is one launch.  Each
// item writes one float64 partial (block reduction); a second kernel sums
// the partials of each (surface, candidate) in a fixed order, so costs are
// deterministic.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/catsurf_b200.h"
#include "errors.h"

namespace {

struct RotSurface {
    const float* src_points;     // [n_src][3]
    const double* src_values;    // [n_src]
    const float* triangles;      // [n_tri][9] target triangle corners
    const int* faces;            // [n_tri][3]
    const double* tgt_values;    // [n_target_points]
    const int* grid_offsets;     // [G^3 + 1]
    const int* grid_faces;       // CSR faces
    const float* matrices;       // [n_candidates][9] column-major
    const float* records;        // [n_tri][kRecordFloats] triangle records or null
    double* partials;            // [n_candidates][tiles]
    int n_src;
    int grid_size;
    int n_candidates;
    int n_features;              // >= 1; values are feature-major
    int n_tgt_points;            // feature stride of tgt_values
    int tiles;                   // ceil(n_src / tile)
    long long item_begin;        // first flat work item of this surface
};

// Up to kInlineSurfaces surfaces travel to the kernels as a launch parameter (no host-to-device
// copy per call); more are read from the scratch copy.
constexpr int kInlineSurfaces = 4;
struct SurfaceTable {
    RotSurface s[kInlineSurfaces];
    long long cost_off[kInlineSurfaces];
};

__device__ __forceinline__ float dot3(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

__device__ __forceinline__ void cross3(const float* a, const float* b, float* out) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ void sub3(const float* a, const float* b, float* out) {
    out[0] = a[0] - b[0];
    out[1] = a[1] - b[1];
    out[2] = a[2] - b[2];
}

// Closest point of q on segment [first, second] (surface_rotation.py:315-333).
__device__ __forceinline__ float segment(const float* q, const float* first, const float* second, float* closest) {
    float dir[3], off[3];
    sub3(second, first, dir);
    sub3(q, first, off);
    const float den = dot3(dir, dir);
    float alpha = den != 0.0f ? dot3(off, dir) / den : 0.0f;
    alpha = alpha < 0.0f ? 0.0f : (alpha > 1.0f ? 1.0f : alpha);
    for (int k = 0; k < 3; ++k) closest[k] = first[k] + alpha * dir[k];
    float d[3];
    sub3(q, closest, d);
    return dot3(d, d);
}

// Candidate distance and closest point for one triangle (354-440).
__device__ __forceinline__ float candidate(const float* q, const float* t, float* point) {
    const float* p0 = t;
    const float* p1 = t + 3;
    const float* p2 = t + 6;
    float ea[3], eb[3], n[3], off[3];
    sub3(p1, p0, ea);
    sub3(p2, p0, eb);
    cross3(ea, eb, n);
    const float nsq = dot3(n, n);
    sub3(p0, q, off);
    const float plane_t = nsq != 0.0f ? dot3(off, n) / nsq : 0.0f;
    float proj[3], po[3];
    for (int k = 0; k < 3; ++k) proj[k] = q[k] + plane_t * n[k];
    sub3(proj, p0, po);
    const float xx = dot3(ea, ea), xy = dot3(ea, eb), xv = dot3(ea, po), yy = dot3(eb, eb), yv = dot3(eb, po);
    const float den = xx * yy - xy * xy;
    const float xpos = den != 0.0f ? (xv * yy - yv * xy) / den : 0.0f;
    const float ypos = den != 0.0f ? (yv * xx - xv * xy) / den : 0.0f;
    const float lo = -1.0e-3f, hi = static_cast<float>(1.0 + 1.0e-3);
    const float s = xpos + ypos;
    const bool inside = den != 0.0f && xpos >= lo && xpos <= hi && ypos >= lo && ypos <= hi && s >= lo && s <= hi;
    if (inside) {
        for (int k = 0; k < 3; ++k) point[k] = proj[k];
        return plane_t * plane_t * nsq;
    }
    float d[3][3];
    float vd[3];
    for (int v = 0; v < 3; ++v) {
        sub3(q, t + 3 * v, d[v]);
        vd[v] = dot3(d[v], d[v]);
    }
    int cv = 0;  // first minimum
    if (vd[1] < vd[cv]) cv = 1;
    if (vd[2] < vd[cv]) cv = 2;
    const float* closest = t + 3 * cv;
    const float* prev = t + 3 * ((cv + 2) % 3);
    const float* next = t + 3 * ((cv + 1) % 3);
    float c1[3], c2[3];
    const float d1 = segment(q, prev, closest, c1);
    const float d2 = segment(q, closest, next, c2);
    const bool first = d1 < d2;
    for (int k = 0; k < 3; ++k) point[k] = first ? c1[k] : c2[k];
    return first ? d1 : d2;
}

// The same candidate from a precomputed triangle record (corners, n, n.n,
// ea.ea, ea.eb, eb.eb; see csg_rotation_triangle_records): four 16-byte loads
// instead of nine scalar ones, and the cross and dot products of the corners
// read instead of formed.  Every value is the one candidate() forms, so the
// result is the same bit for bit.
__device__ __forceinline__ float candidate_record(const float* q, const float* rec, float* point) {
    const float4* r4 = reinterpret_cast<const float4*>(rec);
    const float4 r0 = __ldg(r4), r1 = __ldg(r4 + 1), r2 = __ldg(r4 + 2), r3 = __ldg(r4 + 3);
    const float t[9] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x};
    const float n[3] = {r2.y, r2.z, r2.w};
    const float nsq = r3.x, xx = r3.y, xy = r3.z, yy = r3.w;
    const float* p0 = t;
    float ea[3], eb[3], off[3];
    sub3(t + 3, p0, ea);
    sub3(t + 6, p0, eb);
    sub3(p0, q, off);
    const float plane_t = nsq != 0.0f ? dot3(off, n) / nsq : 0.0f;
    float proj[3], po[3];
    for (int k = 0; k < 3; ++k) proj[k] = q[k] + plane_t * n[k];
    sub3(proj, p0, po);
    const float xv = dot3(ea, po), yv = dot3(eb, po);
    const float den = xx * yy - xy * xy;
    const float xpos = den != 0.0f ? (xv * yy - yv * xy) / den : 0.0f;
    const float ypos = den != 0.0f ? (yv * xx - xv * xy) / den : 0.0f;
    const float lo = -1.0e-3f, hi = static_cast<float>(1.0 + 1.0e-3);
    const float s = xpos + ypos;
    const bool inside = den != 0.0f && xpos >= lo && xpos <= hi && ypos >= lo && ypos <= hi && s >= lo && s <= hi;
    if (inside) {
        for (int k = 0; k < 3; ++k) point[k] = proj[k];
        return plane_t * plane_t * nsq;
    }
    float d[3][3];
    float vd[3];
    for (int v = 0; v < 3; ++v) {
        sub3(q, t + 3 * v, d[v]);
        vd[v] = dot3(d[v], d[v]);
    }
    int cv = 0;  // first minimum
    if (vd[1] < vd[cv]) cv = 1;
    if (vd[2] < vd[cv]) cv = 2;
    const float* closest = t + 3 * cv;
    const float* prev = t + 3 * ((cv + 2) % 3);
    const float* next = t + 3 * ((cv + 1) % 3);
    float c1[3], c2[3];
    const float d1 = segment(q, prev, closest, c1);
    const float d2 = segment(q, closest, next, c2);
    const bool first = d1 < d2;
    for (int k = 0; k < 3; ++k) point[k] = first ? c1[k] : c2[k];
    return first ? d1 : d2;
}

// Per-triangle record (kRecordFloats floats): corners, normal, n.n and the edge Gram
// terms (the float32 values candidate() forms), then a bounding sphere: centre and a
// radius that also covers the closest-polygon test's 1e-3 parametric tolerance.
constexpr int kRecordFloats = 20;
constexpr int kMaxCompact = 64;  // candidates per cell whose reaches the cost scan keeps
static_assert(kMaxCompact <= 64, "the survivors of a cell are one 64-bit mask");

__global__ void k_triangle_records(const float* __restrict__ tri, int n, float* __restrict__ rec) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    const float* t = tri + 9LL * f;
    float ea[3], eb[3], nv[3];
    sub3(t + 3, t, ea);
    sub3(t + 6, t, eb);
    cross3(ea, eb, nv);
    float* r = rec + static_cast<long long>(kRecordFloats) * f;
    for (int k = 0; k < 9; ++k) r[k] = t[k];
    for (int k = 0; k < 3; ++k) r[9 + k] = nv[k];
    r[12] = dot3(nv, nv);
    r[13] = dot3(ea, ea);
    r[14] = dot3(ea, eb);
    r[15] = dot3(eb, eb);
    double c[3], radius = 0.0, edge = 0.0;
    for (int k = 0; k < 3; ++k) c[k] = (static_cast<double>(t[k]) + t[3 + k] + t[6 + k]) / 3.0;
    for (int v = 0; v < 3; ++v) {
        double dc = 0.0, de = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double a = t[3 * v + k] - c[k], b = t[3 * ((v + 1) % 3) + k] - static_cast<double>(t[3 * v + k]);
            dc += a * a;
            de += b * b;
        }
        radius = fmax(radius, sqrt(dc));
        edge = fmax(edge, sqrt(de));
    }
    // a point accepted by the tolerant test lies within 1e-3 of the triangle in parametric
    // coordinates, i.e. within 2e-3 x the longest edge of it
    for (int k = 0; k < 3; ++k) r[16 + k] = static_cast<float>(c[k]);
    const double scale = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    r[19] = static_cast<float>((radius + 4.0e-3 * edge) * 1.001 + 1.0e-6 * scale);
}

// Lower bound of the distance from q to every point the test can return for a record's
// triangle (0 when q is inside the bounding sphere).
__device__ __forceinline__ float record_reach(const float* q, const float* rec) {
    const float4 b = __ldg(reinterpret_cast<const float4*>(rec) + 4);
    const float dx = q[0] - b.x, dy = q[1] - b.y, dz = q[2] - b.z;
    const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
    return dist > b.w ? dist - b.w : 0.0f;
}

// Barycentric weights of `point` in triangle t (surface_rotation.py:335-352).
__device__ __forceinline__ void barycentric(const float* point, const float* t, float w[3]) {
    const int order[3][3] = {{1, 2, 0}, {2, 0, 1}, {0, 1, 2}};
    for (int k = 0; k < 3; ++k) {
        const float* a = t + 3 * order[k][0];
        const float* b = t + 3 * order[k][1];
        const float* c = t + 3 * order[k][2];
        float fo[3], hz[3], up[3], n[3], vert[3];
        sub3(point, a, fo);
        sub3(b, a, hz);
        sub3(c, a, up);
        cross3(hz, up, n);
        cross3(n, hz, vert);
        w[k] = dot3(fo, vert) / dot3(up, vert);
    }
}

template <int TILE>
__global__ void __launch_bounds__(TILE) k_rotation_cost(const __grid_constant__ SurfaceTable table,
                                                        const RotSurface* __restrict__ many, int n_surfaces,
                                                        long long n_items, int* __restrict__ error) {
    __shared__ double red[TILE / 32];
    const RotSurface* surfaces = n_surfaces <= kInlineSurfaces ? table.s : many;
    for (long long item = blockIdx.x; item < n_items; item += gridDim.x) {
        // locate the surface of this item (few surfaces: linear scan)
        int s = 0;
        while (s + 1 < n_surfaces && surfaces[s + 1].item_begin <= item) ++s;
        const RotSurface& S = surfaces[s];
        const long long local = item - S.item_begin;
        const int cand = static_cast<int>(local / S.tiles);
        const int tile = static_cast<int>(local - static_cast<long long>(cand) * S.tiles);
        const int i = tile * TILE + threadIdx.x;
        double contrib = 0.0;
        if (i < S.n_src) {
            const float* m = S.matrices + 9 * cand;
            const float px = S.src_points[3 * i], py = S.src_points[3 * i + 1], pz = S.src_points[3 * i + 2];
            float q[3];
            for (int j = 0; j < 3; ++j) q[j] = (px * m[3 * j] + py * m[3 * j + 1]) + pz * m[3 * j + 2];
            const int G = S.grid_size;
            const float half = static_cast<float>(G / 2.0);
            int cell[3];
            for (int k = 0; k < 3; ++k) {
                int c = static_cast<int>(floorf((q[k] + 1.0f) * half));
                cell[k] = c < 0 ? 0 : (c > G - 1 ? G - 1 : c);
            }
            const long long cid = cell[0] + static_cast<long long>(G) * (cell[1] + static_cast<long long>(G) * cell[2]);
            const int begin = S.grid_offsets[cid], end = S.grid_offsets[cid + 1];
            if (begin >= end) {
                atomicExch(error, CSG_ERR_COVERAGE);
            } else {
                float best = INFINITY;
                int best_face = -1;
                float best_point[3] = {0.0f, 0.0f, 0.0f};
                // With records: the candidate of least reach gives a distance d0 that the first
                // minimum cannot exceed, and a candidate whose reach is clearly above sqrt(d0)
                // cannot be it, so the scan skips it; every other candidate is tested in cell
                // order exactly as without the bound. Cells of at most kMaxCompact candidates
                // keep the reaches of the first pass and test the survivors of a bit mask, so
                // the threads of a warp loop over their own short lists.
                const int count = end - begin;
                const bool compact = S.records != nullptr && count <= kMaxCompact;
                float reach[kMaxCompact];
                float limit = INFINITY;
                if (S.records) {
                    float least = INFINITY;
                    int pick = -1;
                    for (int k = 0; k < count; ++k) {
                        const int f = S.grid_faces[begin + k];
                        const float r = record_reach(q, S.records + kRecordFloats * static_cast<long long>(f));
                        if (compact) reach[k] = r;
                        if (r < least) {
                            least = r;
                            pick = f;
                        }
                    }
                    if (pick >= 0) {
                        float point[3];
                        const float d0 = candidate_record(q, S.records + kRecordFloats * static_cast<long long>(pick), point);
                        // margins far above float32 rounding of the distances, relative to the
                        // coordinates' scale
                        const float scale = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                        if (d0 >= 0.0f && d0 < INFINITY) limit = sqrtf(d0) * 1.0001f + 1.0e-6f * scale;
                    }
                }
                auto test = [&](int f) {
                    float point[3];
                    const float d = S.records ? candidate_record(q, S.records + kRecordFloats * static_cast<long long>(f), point)
                                              : candidate(q, S.triangles + 9 * static_cast<long long>(f), point);
                    if (d < best) {
                        best = d;
                        best_face = f;
                        best_point[0] = point[0];
                        best_point[1] = point[1];
                        best_point[2] = point[2];
                    }
                };
                if (compact) {
                    unsigned long long live = 0;
                    for (int k = 0; k < count; ++k)
                        if (!(reach[k] > limit)) live |= 1ull << k;
                    while (live) {
                        const int k = __ffsll(static_cast<long long>(live)) - 1;
                        live &= live - 1;
                        test(S.grid_faces[begin + k]);
                    }
                } else {
                    for (int k = begin; k < end; ++k) {
                        const int f = S.grid_faces[k];
                        if (S.records && record_reach(q, S.records + kRecordFloats * static_cast<long long>(f)) > limit)
                            continue;
                        test(f);
                    }
                }
                if (best_face < 0) {  // every candidate produced NaN
                    best_face = S.grid_faces[begin];
                    candidate(q, S.triangles + 9 * static_cast<long long>(best_face), best_point);
                }
                float w[3];
                barycentric(best_point, S.triangles + 9 * static_cast<long long>(best_face), w);
                const int* fv = S.faces + 3 * static_cast<long long>(best_face);
                for (int f = 0; f < S.n_features; ++f) {
                    const double* tv = S.tgt_values + static_cast<long long>(f) * S.n_tgt_points;
                    const double sampled = (tv[fv[0]] * static_cast<double>(w[0]) +
                                            tv[fv[1]] * static_cast<double>(w[1])) +
                                           tv[fv[2]] * static_cast<double>(w[2]);
                    const double diff = S.src_values[static_cast<long long>(f) * S.n_src + i] - sampled;
                    contrib = contrib + diff * diff;
                }
            }
        }
        // fixed-order block reduction: warp tree, then warp 0 over warp sums
        for (int off = 16; off > 0; off >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = contrib;
        __syncthreads();
        if (threadIdx.x < 32) {
            double v = threadIdx.x < TILE / 32 ? red[threadIdx.x] : 0.0;
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (threadIdx.x == 0) S.partials[static_cast<long long>(cand) * S.tiles + tile] = v;
        }
        __syncthreads();
    }
}

__global__ void k_rotation_finalize(const __grid_constant__ SurfaceTable table, const RotSurface* __restrict__ many,
                                    int n_surfaces, double* __restrict__ costs, const long long* __restrict__ many_offsets) {
    const int s = blockIdx.y;
    if (s >= n_surfaces) return;
    const bool inline_table = n_surfaces <= kInlineSurfaces;
    const RotSurface* surfaces = inline_table ? table.s : many;
    const long long* cost_offsets = inline_table ? table.cost_off : many_offsets;
    const RotSurface& S = surfaces[s];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= S.n_candidates) return;
    // the partials in tile order, loaded kAhead at a time before they are added (the
    // additions stay in that order; the loads no longer wait on one another)
    constexpr int kAhead = 32;
    double total = 0.0;
    const double* p = S.partials + static_cast<long long>(c) * S.tiles;
    int t = 0;
    for (; t + kAhead <= S.tiles; t += kAhead) {
        double part[kAhead];
#pragma unroll
        for (int j = 0; j < kAhead; ++j) part[j] = p[t + j];
#pragma unroll
        for (int j = 0; j < kAhead; ++j) total += part[j];
    }
    for (; t < S.tiles; ++t) total += p[t];
    costs[cost_offsets[s] + c] = total;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// ---------------------------------------------------- device grid build
// Same cells as csg_rotation_grid_build (bounding box of each triangle in
// cells of size 2 / G over [-1, 1]^3, +/- margin, clamped); counts by
// atomics, a two-level scan, an atomic fill, then every cell's list sorted
// ascending so the candidate order (and the first-minimum rule) is the
// host builder's.

constexpr int kScan = 1024;

__device__ __forceinline__ void face_cells(const double* pts, const int* faces, int f, int G, int margin, int lo[3],
                                           int hi[3]) {
    const double cell = 2.0 / static_cast<double>(G);
    const int v0 = faces[3 * f], v1 = faces[3 * f + 1], v2 = faces[3 * f + 2];
    for (int k = 0; k < 3; ++k) {
        const double a = pts[3 * v0 + k], b = pts[3 * v1 + k], c = pts[3 * v2 + k];
        const double mn = fmin(fmin(a, b), c), mx = fmax(fmax(a, b), c);
        const long long l = static_cast<long long>(floor((mn + 1.0) / cell)) - margin;
        const long long h = static_cast<long long>(floor((mx + 1.0) / cell)) + margin;
        lo[k] = static_cast<int>(l < 0 ? 0 : (l > G - 1 ? G - 1 : l));
        hi[k] = static_cast<int>(h < 0 ? 0 : (h > G - 1 ? G - 1 : h));
    }
}

__global__ void k_rgrid_count(const double* __restrict__ pts, const int* __restrict__ faces, int n_faces, int G,
                              int margin, int* __restrict__ counts) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    int lo[3], hi[3];
    face_cells(pts, faces, f, G, margin, lo, hi);
    for (int z = lo[2]; z <= hi[2]; ++z)
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int x = lo[0]; x <= hi[0]; ++x)
                atomicAdd(counts + x + static_cast<long long>(G) * (y + static_cast<long long>(G) * z) + 1, 1);
}

__global__ void k_rgrid_scan_block(int* __restrict__ data, int n, int* __restrict__ sums) {
    __shared__ int buf[kScan];
    const int i = blockIdx.x * kScan + threadIdx.x;
    buf[threadIdx.x] = i < n ? data[i] : 0;
    __syncthreads();
    for (int off = 1; off < kScan; off <<= 1) {
        const int v = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
        __syncthreads();
        buf[threadIdx.x] += v;
        __syncthreads();
    }
    if (i < n) data[i] = buf[threadIdx.x];
    if (threadIdx.x == kScan - 1) sums[blockIdx.x] = buf[threadIdx.x];
}

__global__ void k_rgrid_scan_sums(int* __restrict__ sums, int nblocks) {
    __shared__ int buf[kScan];
    int carry = 0;
    for (int base = 0; base < nblocks; base += kScan) {
        const int i = base + threadIdx.x;
        const int own = i < nblocks ? sums[i] : 0;
        buf[threadIdx.x] = own;
        __syncthreads();
        for (int off = 1; off < kScan; off <<= 1) {
            const int v = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += v;
            __syncthreads();
        }
        if (i < nblocks) sums[i] = carry + buf[threadIdx.x] - own;
        const int total = buf[kScan - 1];
        __syncthreads();
        carry += total;
    }
}

__global__ void k_rgrid_scan_add(int* __restrict__ data, int n, const int* __restrict__ sums, int* __restrict__ cursor) {
    const int i = blockIdx.x * kScan + threadIdx.x;
    if (i >= n) return;
    const int v = data[i] + sums[blockIdx.x];
    data[i] = v;
    if (cursor && i + 1 < n) cursor[i] = v;
}

__global__ void k_rgrid_fill(const double* __restrict__ pts, const int* __restrict__ faces, int n_faces, int G,
                             int margin, int* __restrict__ cursor, int* __restrict__ cell_faces) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    int lo[3], hi[3];
    face_cells(pts, faces, f, G, margin, lo, hi);
    for (int z = lo[2]; z <= hi[2]; ++z)
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int x = lo[0]; x <= hi[0]; ++x)
                cell_faces[atomicAdd(cursor + x + static_cast<long long>(G) * (y + static_cast<long long>(G) * z), 1)] = f;
}

// Insertion sort of each cell's (short) face list.
__global__ void k_rgrid_sort(const int* __restrict__ offsets, long long n_cells, int* __restrict__ cell_faces) {
    const long long c = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const int b = offsets[c], e = offsets[c + 1];
    for (int i = b + 1; i < e; ++i) {
        const int key = cell_faces[i];
        int j = i - 1;
        while (j >= b && cell_faces[j] > key) {
            cell_faces[j + 1] = cell_faces[j];
            --j;
        }
        cell_faces[j + 1] = key;
    }
}

}  // namespace

extern "C" {

int csg_rotation_grid_build(const double* points, int n_points, const int32_t* faces, int n_faces, int grid_size,
                            int margin, int32_t* offsets, int32_t* cell_faces, long long capacity, long long* count) {
    if (!points || !faces || n_points < 1 || n_faces < 1 || grid_size < 4 || margin < 0 || !offsets || !count)
        return csg::fail(CSG_ERR_ARG, "rotation grid: bad arguments (grid_size >= 4, margin >= 0)");
    if (static_cast<long long>(grid_size) * grid_size * grid_size >= (1LL << 31))
        return csg::fail(CSG_ERR_ARG, "rotation grid: grid_size too large");
    const int G = grid_size;
    const double cell = 2.0 / static_cast<double>(G);
    std::vector<int> lo(3 * static_cast<size_t>(n_faces)), hi(3 * static_cast<size_t>(n_faces));
    const long long ncell = static_cast<long long>(G) * G * G;
    std::vector<long long> counts(ncell + 1, 0);
    for (int f = 0; f < n_faces; ++f) {
        for (int k = 0; k < 3; ++k) {
            const int v0 = faces[3 * f], v1 = faces[3 * f + 1], v2 = faces[3 * f + 2];
            if (v0 < 0 || v1 < 0 || v2 < 0 || v0 >= n_points || v1 >= n_points || v2 >= n_points)
                return csg::fail(CSG_ERR_TOPOLOGY, "rotation grid: face %d references a missing point", f);
            const double a = points[3 * v0 + k], b = points[3 * v1 + k], c = points[3 * v2 + k];
            const double mn = std::min(std::min(a, b), c), mx = std::max(std::max(a, b), c);
            long long l = static_cast<long long>(std::floor((mn + 1.0) / cell)) - margin;
            long long h = static_cast<long long>(std::floor((mx + 1.0) / cell)) + margin;
            lo[3 * f + k] = static_cast<int>(std::min<long long>(std::max<long long>(l, 0), G - 1));
            hi[3 * f + k] = static_cast<int>(std::min<long long>(std::max<long long>(h, 0), G - 1));
        }
        for (int z = lo[3 * f + 2]; z <= hi[3 * f + 2]; ++z)
            for (int y = lo[3 * f + 1]; y <= hi[3 * f + 1]; ++y)
                for (int x = lo[3 * f]; x <= hi[3 * f]; ++x) counts[x + static_cast<long long>(G) * (y + static_cast<long long>(G) * z) + 1]++;
    }
    for (long long c = 0; c < ncell; ++c) counts[c + 1] += counts[c];
    *count = counts[ncell];
    if (counts[ncell] >= (1LL << 31)) return csg::fail(CSG_ERR_ARG, "rotation grid: more than 2^31 entries");
    for (long long c = 0; c <= ncell; ++c) offsets[c] = static_cast<int32_t>(counts[c]);
    if (!cell_faces) return CSG_OK;  // size query
    if (capacity < counts[ncell]) return csg::fail(CSG_ERR_ARG, "rotation grid: capacity %lld < %lld", capacity, counts[ncell]);
    std::vector<long long> fill(counts.begin(), counts.end() - 1);
    for (int f = 0; f < n_faces; ++f)
        for (int z = lo[3 * f + 2]; z <= hi[3 * f + 2]; ++z)
            for (int y = lo[3 * f + 1]; y <= hi[3 * f + 1]; ++y)
                for (int x = lo[3 * f]; x <= hi[3 * f]; ++x)
                    cell_faces[fill[x + static_cast<long long>(G) * (y + static_cast<long long>(G) * z)]++] = f;
    return CSG_OK;
}

size_t csg_rotation_scratch_bytes(int n_surfaces, const int* n_src, const int* n_candidates, int tile) {
    if (n_surfaces < 1 || !n_src || !n_candidates || (tile != 128 && tile != 256 && tile != 512)) return 0;
    size_t bytes = align256(sizeof(RotSurface) * n_surfaces) + align256(sizeof(long long) * n_surfaces) + 256;
    for (int s = 0; s < n_surfaces; ++s) {
        const size_t tiles = (static_cast<size_t>(n_src[s]) + tile - 1) / tile;
        bytes += align256(sizeof(double) * tiles * static_cast<size_t>(n_candidates[s]));
    }
    return bytes;
}

int csg_rotation_cost_batch(int n_surfaces, const csg_rotation_surface* surfaces, double* costs, int tile,
                            int n_ctas, void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    if (n_surfaces < 1 || !surfaces || !costs || !scratch) return csg::fail(CSG_ERR_ARG, "rotation cost: bad arguments");
    if (tile <= 0) tile = 256;
    if (tile != 128 && tile != 256 && tile != 512) return csg::fail(CSG_ERR_ARG, "rotation cost: tile must be 128, 256 or 512");
    std::vector<int> ns(n_surfaces), nc(n_surfaces);
    for (int s = 0; s < n_surfaces; ++s) {
        const csg_rotation_surface& in = surfaces[s];
        if (!in.src_points || !in.src_values || !in.triangles || !in.faces || !in.tgt_values || !in.grid_offsets ||
            !in.grid_faces || !in.matrices || in.n_src < 1 || in.n_candidates < 1 || in.grid_size < 4 ||
            in.n_features < 0 || (in.n_features > 1 && in.n_tgt_points < 1))
            return csg::fail(CSG_ERR_ARG, "rotation cost: surface %d is incomplete", s);
        if (reinterpret_cast<uintptr_t>(in.records) % 16 != 0)
            return csg::fail(CSG_ERR_ARG, "rotation cost: surface %d's triangle records are not 16-byte aligned", s);
        ns[s] = in.n_src;
        nc[s] = in.n_candidates;
    }
    if (scratch_bytes < csg_rotation_scratch_bytes(n_surfaces, ns.data(), nc.data(), tile))
        return csg::fail(CSG_ERR_ARG, "rotation cost: scratch too small");
    char* base = static_cast<char*>(scratch);
    RotSurface* d_surf = reinterpret_cast<RotSurface*>(base);
    size_t used = align256(sizeof(RotSurface) * n_surfaces);
    long long* d_off = reinterpret_cast<long long*>(base + used);
    used += align256(sizeof(long long) * n_surfaces);
    int* d_err = reinterpret_cast<int*>(base + used);
    used += 256;
    std::vector<RotSurface> host(n_surfaces);
    std::vector<long long> cost_off(n_surfaces);
    long long items = 0, coff = 0;
    int max_c = 0;
    for (int s = 0; s < n_surfaces; ++s) {
        const csg_rotation_surface& in = surfaces[s];
        RotSurface& r = host[s];
        r.src_points = in.src_points;
        r.src_values = in.src_values;
        r.triangles = in.triangles;
        r.faces = in.faces;
        r.tgt_values = in.tgt_values;
        r.grid_offsets = in.grid_offsets;
        r.grid_faces = in.grid_faces;
        r.matrices = in.matrices;
        r.records = in.records;
        r.n_src = in.n_src;
        r.grid_size = in.grid_size;
        r.n_candidates = in.n_candidates;
        r.n_features = in.n_features > 1 ? in.n_features : 1;
        r.n_tgt_points = in.n_features > 1 ? in.n_tgt_points : 0;
        r.tiles = (in.n_src + tile - 1) / tile;
        r.partials = reinterpret_cast<double*>(base + used);
        used += align256(sizeof(double) * static_cast<size_t>(r.tiles) * r.n_candidates);
        r.item_begin = items;
        items += static_cast<long long>(r.tiles) * r.n_candidates;
        cost_off[s] = coff;
        coff += r.n_candidates;
        max_c = std::max(max_c, r.n_candidates);
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    SurfaceTable table{};
    if (n_surfaces <= kInlineSurfaces) {
        for (int s = 0; s < n_surfaces; ++s) {
            table.s[s] = host[s];
            table.cost_off[s] = cost_off[s];
        }
    } else {
        CSG_CUDA_CHECK(cudaMemcpyAsync(d_surf, host.data(), sizeof(RotSurface) * n_surfaces, cudaMemcpyHostToDevice, st));
        CSG_CUDA_CHECK(cudaMemcpyAsync(d_off, cost_off.data(), sizeof(long long) * n_surfaces, cudaMemcpyHostToDevice, st));
    }
    CSG_CUDA_CHECK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    int device = 0, sms = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const long long want = n_ctas > 0 ? n_ctas : static_cast<long long>(sms) * (2048 / tile);
    const unsigned blocks = static_cast<unsigned>(std::min<long long>(std::max<long long>(1, want), items));
    switch (tile) {
        case 128: (csg::note_launch(), k_rotation_cost<128><<<blocks, 128, 0, st>>>(table, d_surf, n_surfaces, items, d_err)); break;
        case 512: (csg::note_launch(), k_rotation_cost<512><<<blocks, 512, 0, st>>>(table, d_surf, n_surfaces, items, d_err)); break;
        default: (csg::note_launch(), k_rotation_cost<256><<<blocks, 256, 0, st>>>(table, d_surf, n_surfaces, items, d_err)); break;
    }
    (csg::note_launch(), k_rotation_finalize<<<dim3((max_c + 127) / 128, n_surfaces), 128, 0, st>>>(table, d_surf, n_surfaces, costs, d_off));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

size_t csg_rotation_grid_scratch_bytes(int grid_size) {
    if (grid_size < 4 || static_cast<long long>(grid_size) * grid_size * grid_size >= (1LL << 31)) return 0;
    const long long cells = static_cast<long long>(grid_size) * grid_size * grid_size;
    return align256(sizeof(int) * static_cast<size_t>(cells)) + align256(sizeof(int) * ((cells + 1) / kScan + 2));
}

int csg_rotation_grid_build_device(const double* points, int n_points, const int32_t* faces, int n_faces,
                                   int grid_size, int margin, int32_t* offsets, int32_t* cell_faces,
                                   long long capacity, long long* count, void* scratch, size_t scratch_bytes,
                                   csg_stream_t stream) {
    if (!points || !faces || n_points < 1 || n_faces < 1 || grid_size < 4 || margin < 0 || !offsets || !count ||
        !scratch)
        return csg::fail(CSG_ERR_ARG, "rotation grid (device): bad arguments (grid_size >= 4, margin >= 0)");
    if (scratch_bytes < csg_rotation_grid_scratch_bytes(grid_size))
        return csg::fail(CSG_ERR_ARG, "rotation grid (device): scratch too small");
    const int G = grid_size;
    const long long cells = static_cast<long long>(G) * G * G;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(scratch);
    int* cursor = reinterpret_cast<int*>(base);
    int* sums = reinterpret_cast<int*>(base + align256(sizeof(int) * static_cast<size_t>(cells)));
    CSG_CUDA_CHECK(cudaMemsetAsync(offsets, 0, sizeof(int32_t) * static_cast<size_t>(cells + 1), st));
    const unsigned fb = static_cast<unsigned>((n_faces + 255) / 256);
    (csg::note_launch(), k_rgrid_count<<<fb, 256, 0, st>>>(points, faces, n_faces, G, margin, offsets));
    const int n = static_cast<int>(cells + 1);
    const int nblocks = (n + kScan - 1) / kScan;
    (csg::note_launch(), k_rgrid_scan_block<<<nblocks, kScan, 0, st>>>(offsets, n, sums));
    (csg::note_launch(), k_rgrid_scan_sums<<<1, kScan, 0, st>>>(sums, nblocks));
    (csg::note_launch(), k_rgrid_scan_add<<<nblocks, kScan, 0, st>>>(offsets, n, sums, cursor));
    int total = 0;
    CSG_CUDA_CHECK(cudaMemcpyAsync(&total, offsets + cells, sizeof(int), cudaMemcpyDeviceToHost, st));
    CSG_CUDA_CHECK(cudaStreamSynchronize(st));
    *count = total;
    if (!cell_faces) return CSG_OK;  // size query
    if (capacity < total) return csg::fail(CSG_ERR_ARG, "rotation grid (device): capacity %lld < %d", capacity, total);
    (csg::note_launch(), k_rgrid_fill<<<fb, 256, 0, st>>>(points, faces, n_faces, G, margin, cursor, cell_faces));
    (csg::note_launch(), k_rgrid_sort<<<static_cast<unsigned>((cells + 255) / 256), 256, 0, st>>>(offsets, cells,
                                                                                                 cell_faces));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_rotation_triangle_records(const float* triangles, int n_tri, float* records, csg_stream_t stream) {
    if (!triangles || !records || n_tri < 1) return csg::fail(CSG_ERR_ARG, "triangle records: bad arguments");
    if (reinterpret_cast<uintptr_t>(records) % 16 != 0)
        return csg::fail(CSG_ERR_ARG, "triangle records: records must be 16-byte aligned");
    (csg::note_launch(), k_triangle_records<<<static_cast<unsigned>((n_tri + 255) / 256), 256, 0,
                                              reinterpret_cast<cudaStream_t>(stream)>>>(triangles, n_tri, records));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

size_t csg_rotation_status_offset(int n_surfaces) {
    if (n_surfaces < 1) return 0;
    return align256(sizeof(RotSurface) * n_surfaces) + align256(sizeof(long long) * n_surfaces);
}

int csg_rotation_status(const void* scratch, int n_surfaces, csg_stream_t stream, int* status) {
    if (!scratch || !status || n_surfaces < 1) return csg::fail(CSG_ERR_ARG, "rotation status: bad arguments");
    const size_t off = align256(sizeof(RotSurface) * n_surfaces) + align256(sizeof(long long) * n_surfaces);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    CSG_CUDA_CHECK(cudaMemcpyAsync(status, static_cast<const char*>(scratch) + off, sizeof(int), cudaMemcpyDeviceToHost, st));
    CSG_CUDA_CHECK(cudaStreamSynchronize(st));
    return CSG_OK;
}

int csg_rotation_cost_host(const csg_rotation_surface* surface, const float* matrices_host, float* matrices_device,
                           void* readback_host, int tile, void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    if (!surface || !matrices_host || !matrices_device || !readback_host || !scratch)
        return csg::fail(CSG_ERR_ARG, "rotation cost (host): bad arguments");
    const int count = surface->n_candidates;
    if (count < 1 || count > CSG_ROTATION_HOST_MAX_CANDIDATES)
        return csg::fail(CSG_ERR_ARG, "rotation cost (host): %d candidates (1 to %d; use csg_rotation_cost_batch)",
                         count, CSG_ROTATION_HOST_MAX_CANDIDATES);
    // the status word's 256-byte slot in the scratch holds the costs behind it, so one
    // copy brings both back
    char* slot = static_cast<char*>(scratch) + csg_rotation_status_offset(1);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    csg_rotation_surface local = *surface;
    local.matrices = matrices_device;
    CSG_CUDA_CHECK(cudaMemcpyAsync(matrices_device, matrices_host, sizeof(float) * 9 * static_cast<size_t>(count),
                                   cudaMemcpyHostToDevice, st));
    const int rc = csg_rotation_cost_batch(1, &local, reinterpret_cast<double*>(slot + 8), tile, 0, scratch,
                                           scratch_bytes, stream);
    if (rc) return rc;
    CSG_CUDA_CHECK(cudaMemcpyAsync(readback_host, slot, 8 + sizeof(double) * static_cast<size_t>(count),
                                   cudaMemcpyDeviceToHost, st));
    CSG_CUDA_CHECK(cudaStreamSynchronize(st));
    return CSG_OK;
}

}  // extern "C"
