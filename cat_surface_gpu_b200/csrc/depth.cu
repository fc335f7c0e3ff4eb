// Depth-potential rotation feature (src/cat_surface_gpu/rotation_feature.py)
// on sm_100a: the solve of (L + alpha A) u = (H - mean H) A on the smoothed
// coarse surface, batched over surfaces that share one triangulation.
//
// Setup (three plain kernels):
//   k_depth_faces     per face: the stable-normal terms (_stable_normals
//                     37-74), the mixed Voronoi contributions (77-128) and
//                     the cotangent dots (_system_entries 131-171);
//   k_depth_vertices  per vertex: normal, area, system row, diagonal and mean
//                     curvature, gathering over the incidences sorted by
//                     (corner, face) -- the order of the reference's CPU
//                     index_add_ -- so every row sums in the reference's order;
//   k_depth_rhs       per surface: the area-weighted mean-curvature offset,
//                     rhs and |rhs| as blocked sums.
// Solvers:
//   coloured SOR (253-317): a colour sweep is one Gauss-Seidel pass in
//   colour-major vertex order, so the sweeps run as one persistent wavefront
//   launch over that order's schedule (vertex v of sweep s at step
//   s * D + level(v), as the Surf2Sphere kernels), each CTA keeping the rows
//   of its vertices in shared memory;
//   Jacobi-preconditioned CG (189-250): one persistent cooperative launch.
//
// Arithmetic: float64, one rounding per operation (--fmad=false), with the
// torch CPU kernels' fused forms kept: vector_norm accumulates
// fma(x_i, x_i, acc), linalg.cross forms fma(a, b, -(c d)).  Whole-vector sums
// are blocked -- sequential runs of 256 terms, the run sums folded into 32
// lanes (lane l takes runs l, l + 32, ...), then the lanes pairwise (16, 8, 4,
// 2, 1) -- so results do not depend on the launch shape.
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "common.cuh"
#include "errors.h"

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kEps = 2.220446049250313080847263336181640625e-16;
constexpr int kRun = 256;
constexpr int kRec = 12;  // tn[3], w[3], voronoi contribution[3], d23, d13, d12
constexpr int kThreads = 256;
constexpr int kMaxCgBatch = 8;  // surfaces of one CG launch (per-surface scalars stay in registers)

__device__ __forceinline__ double clamp_eps(double x) { return x < kEps ? kEps : x; }  // keeps NaN
__device__ __forceinline__ double dot3(const double* a, const double* b) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
__device__ __forceinline__ double norm3(const double* a) {
    return sqrt(__fma_rn(a[2], a[2], __fma_rn(a[1], a[1], a[0] * a[0])));
}
__device__ __forceinline__ void cross3(const double* a, const double* b, double* o) {
    o[0] = __fma_rn(a[1], b[2], -(a[2] * b[1]));
    o[1] = __fma_rn(a[2], b[0], -(a[0] * b[2]));
    o[2] = __fma_rn(a[0], b[1], -(a[1] * b[0]));
}

// ---------------------------------------------------------------- setup

struct SetupParams {
    const float* geom;  // [batch][n][3]
    const int* faces;
    const int* inc_off;
    const int* inc;
    int n, nf, batch;
    double alpha;
    double* rec;      // [batch][nf][kRec]
    int* col;         // [nnz], shared by the batch
    double* val;      // [batch][nnz]
    double* areas;    // [batch][n]
    double* diag;     // [batch][n]
    double* mc;       // [batch][n]
    double* rhs;      // [batch][n]
    double* rhs_norm; // [batch]
    double* normals;  // nullable [batch][n][3]
    csg::Control* ctl;
    long long nnz;
};

// Index checks: a bad face or incidence records CSG_ERR_TOPOLOGY; every later
// kernel of the solve sees the status and does nothing.
__device__ __forceinline__ void report(csg::Control* ctl, int code) {
    if (atomicCAS(&ctl->status, CSG_OK, code) == CSG_OK) ctl->where = -1;
}
__device__ __forceinline__ bool failed(const csg::Control* ctl) {
    return *reinterpret_cast<const volatile int*>(&ctl->status) != CSG_OK;
}

__global__ void k_depth_faces(SetupParams p) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(p.nf) * p.batch) return;
    const int b = static_cast<int>(i / p.nf), f = static_cast<int>(i % p.nf);
    const float* g = p.geom + 3LL * p.n * b;
    double q[3][3];
    for (int k = 0; k < 3; ++k) {
        long long v = p.faces[3LL * f + k];
        if (v < 0 || v >= p.n) {
            report(p.ctl, CSG_ERR_TOPOLOGY);
            v = 0;
        }
        for (int c = 0; c < 3; ++c) q[k][c] = static_cast<double>(g[3 * v + c]);
    }
    double v1[3], v2[3], v3[3], u1[3], u2[3], u3[3];
    for (int c = 0; c < 3; ++c) {
        v1[c] = q[1][c] - q[0][c];
        v2[c] = q[2][c] - q[1][c];
        v3[c] = q[0][c] - q[2][c];
    }
    const double n1 = clamp_eps(norm3(v1)), n2 = clamp_eps(norm3(v2)), n3 = clamp_eps(norm3(v3));
    for (int c = 0; c < 3; ++c) {
        u1[c] = v1[c] / n1;
        u2[c] = v2[c] / n2;
        u3[c] = v3[c] / n3;
    }
    double c31[3], c23[3], c12[3];
    cross3(u3, u1, c31);
    cross3(u2, u3, c23);
    cross3(u1, u2, c12);
    const double m31 = clamp_eps(norm3(c31)), m23 = clamp_eps(norm3(c23)), m12 = clamp_eps(norm3(c12));
    double* r = p.rec + kRec * (static_cast<long long>(b) * p.nf + f);
    for (int c = 0; c < 3; ++c) r[c] = c12[c] / m12;
    r[3] = (1.0 - dot3(u3, u1)) / m31;
    r[4] = (1.0 - dot3(u1, u2)) / m12;
    r[5] = (1.0 - dot3(u2, u3)) / m23;
    double cr[3];
    cross3(v1, v2, cr);
    const double area = clamp_eps(norm3(cr));
    const double d31 = dot3(v3, v1), d12 = dot3(v1, v2), d23 = dot3(v2, v3);
    const bool bad0 = d31 > 0.0, bad1 = d12 > 0.0, bad2 = d23 > 0.0;
    const double l1 = dot3(v1, v1), l2 = dot3(v2, v2), l3 = dot3(v3, v3), d13 = dot3(v1, v3);
    const double e = 0.125 * area;
    if (bad0 || bad1 || bad2) {
        r[6] = e + (bad0 ? e : 0.0);
        r[7] = e + (bad1 ? e : 0.0);
        r[8] = e + (bad2 ? e : 0.0);
    } else {
        r[6] = -0.125 * (l3 * d12 + l1 * d23) / area + 0.0;
        r[7] = -0.125 * (l2 * d13 + l1 * d23) / area + 0.0;
        r[8] = -0.125 * (l2 * d13 + l3 * d12) / area + 0.0;
    }
    r[9] = d23 / area;
    r[10] = d13 / area;
    r[11] = d12 / area;
}

// Row v: the diagonal entries of its incidences (corner 0, 1, 2 faces, each in
// face order), the off-diagonal blocks (i0,i1) (i1,i0) (i1,i2) (i2,i1) (i0,i2)
// (i2,i0), then alpha * area -- 3 deg + 1 entries from 3 inc_off[v] + v.
__global__ void k_depth_vertices(SetupParams p) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(p.n) * p.batch) return;
    const int b = static_cast<int>(i / p.n), v = static_cast<int>(i % p.n);
    const float* g = p.geom + 3LL * p.n * b;
    const double* rec = p.rec + kRec * static_cast<long long>(b) * p.nf;
    const int k0 = p.inc_off[v], k1 = p.inc_off[v + 1];
    // rows must stay inside the 9 nf + n entries and reference real faces
    bool ok = k0 >= 0 && k0 <= k1 && k1 <= 3 * p.nf;
    for (int k = k0; ok && k < k1; ++k) ok = (p.inc[k] >> 2) < p.nf && (p.inc[k] & 3) < 3 && p.inc[k] >= 0;
    for (int k = k0; ok && k < k1; ++k)
        for (int c = 0; c < 3; ++c) {
            const int w = p.faces[3LL * (p.inc[k] >> 2) + c];
            ok = ok && w >= 0 && w < p.n;
        }
    if (!ok) {
        report(p.ctl, CSG_ERR_TOPOLOGY);
        return;
    }
    double acc[3] = {0.0, 0.0, 0.0}, a = 0.0;
    for (int k = k0; k < k1; ++k) {
        const int f = p.inc[k] >> 2, corner = p.inc[k] & 3;
        const double* r = rec + kRec * static_cast<long long>(f);
        for (int c = 0; c < 3; ++c) acc[c] = acc[c] + r[c] * r[3 + corner];
        a = a + r[6 + corner];
    }
    const double nn = clamp_eps(norm3(acc));
    double nv[3];
    for (int c = 0; c < 3; ++c) nv[c] = acc[c] / nn;
    if (!isfinite(a) || a == 0.0) a = 1.0;
    const long long at = static_cast<long long>(b) * p.n + v;
    if (p.normals)
        for (int c = 0; c < 3; ++c) p.normals[3 * at + c] = nv[c];
    p.areas[at] = a;

    const long long row = 3LL * k0 + v;
    int* col = p.col + row;
    double* val = p.val + static_cast<long long>(b) * p.nnz + row;
    const bool write_col = b == 0;
    int m = 0;
    double d = 0.0, lap[3] = {0.0, 0.0, 0.0};
    auto put = [&](int c, double x, bool laplacian) {
        if (write_col) col[m] = c;
        val[m] = x;
        ++m;
        d = d + (c == v ? x : 0.0);
        if (laplacian)
            for (int k = 0; k < 3; ++k) lap[k] = lap[k] + x * static_cast<double>(g[3LL * c + k]);
    };
    for (int k = k0; k < k1; ++k) {
        const int f = p.inc[k] >> 2, corner = p.inc[k] & 3;
        const double* r = rec + kRec * static_cast<long long>(f);
        put(v, corner == 0 ? -0.5 * (r[9] + r[11]) : (corner == 1 ? -0.5 * (r[10] + r[9]) : -0.5 * (r[11] + r[10])),
            true);
    }
    // (row corner, column corner, record slot) of the six off-diagonal blocks
    constexpr int kBlocks[6][3] = {{0, 1, 9}, {1, 0, 9}, {1, 2, 10}, {2, 1, 10}, {0, 2, 11}, {2, 0, 11}};
#pragma unroll
    for (int q = 0; q < 6; ++q)
        for (int k = k0; k < k1; ++k) {
            const int f = p.inc[k] >> 2, corner = p.inc[k] & 3;
            if (corner != kBlocks[q][0]) continue;
            put(p.faces[3LL * f + kBlocks[q][1]], 0.5 * rec[kRec * static_cast<long long>(f) + kBlocks[q][2]], true);
        }
    put(v, p.alpha * a, false);
    for (int k = 0; k < 3; ++k) lap[k] = lap[k] * 2.0;
    p.diag[at] = clamp_eps(d);
    const double h = 0.5 * dot3(lap, nv) / a;
    p.mc[at] = isfinite(h) ? h : 0.0;
}

// Blocked sum (see the file comment) of term(i), i < n, by one CTA; every
// thread returns the sum.  `runs` is shared scratch of n / kRun + 1 doubles.
template <typename Term>
__device__ double cta_blocked_sum(int n, Term term, double* runs_buf) {
    __shared__ double s_total;
    const int runs = (n + kRun - 1) / kRun;
    for (int r = threadIdx.x; r < runs; r += blockDim.x) {
        double s = 0.0;
        const int e = min(n, (r + 1) * kRun);
        for (int i = r * kRun; i < e; ++i) s = s + term(i);
        runs_buf[r] = s;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        double lane = 0.0;
        for (int r = threadIdx.x; r < runs; r += 32) lane = lane + runs_buf[r];
        for (int off = 16; off >= 1; off >>= 1) lane = lane + __shfl_down_sync(kFull, lane, off);
        if (threadIdx.x == 0) s_total = lane;
    }
    __syncthreads();
    const double total = s_total;
    __syncthreads();
    return total;
}

// One CTA per surface: factor = sum(H A) / sum(A), rhs = (H - factor) A, |rhs|.
__global__ void k_depth_rhs(SetupParams p, double* runs_buf) {
    if (failed(p.ctl)) return;
    const int b = blockIdx.x;
    const long long base = static_cast<long long>(b) * p.n;
    const double* mc = p.mc + base;
    const double* ar = p.areas + base;
    double* rhs = p.rhs + base;
    double* buf = runs_buf + static_cast<long long>(b) * ((p.n + kRun - 1) / kRun + 1);
    const double s_ha = cta_blocked_sum(p.n, [&](int i) { return mc[i] * ar[i]; }, buf);
    const double s_a = cta_blocked_sum(p.n, [&](int i) { return ar[i]; }, buf);
    const double factor = s_ha / s_a;
    for (int i = threadIdx.x; i < p.n; i += blockDim.x) rhs[i] = (mc[i] - factor) * ar[i];
    __syncthreads();
    const double s_rr = cta_blocked_sum(p.n, [&](int i) { return rhs[i] * rhs[i]; }, buf);
    if (threadIdx.x == 0) p.rhs_norm[b] = clamp_eps(sqrt(s_rr));
}

// ---------------------------------------------------------------- SOR

struct SorParams {
    const int* inc_off;  // row v starts at 3 inc_off[v] + v, has 3 deg + 1 entries
    const int* col;
    const double* val;   // [batch][nnz]
    const double* diag;  // [batch][n]
    const double* rhs;   // [batch][n]
    double* x;           // [batch][n]
    const int* order;    // wavefront schedule of the colour-major order
    const int* level_begin;
    const int* level_end;
    csg::Control* ctl;
    long long nnz;
    int n, batch, n_levels, stride, sweeps;
    int max_row, nloc_max;  // shared-memory image (0: rows read from global memory)
    double relaxation;
    unsigned long long timeout_ns;
    unsigned long long* pub;  // dataflow form: x as versioned words, 2 per (surface, vertex)
    int* level_of;            // dataflow form: the schedule level of every vertex
};

__device__ __forceinline__ int owned_below(int bound, int c, int nc) { return bound > c ? (bound - c + nc - 1) / nc : 0; }

// Row sum of one surface by a group of G lanes.  Lane j loads and multiplies
// entries j, j + G, ..., j + (32 / G - 1) G of a block of 32 entries first (all
// of a row's gathers in flight together), then the products are added in entry
// order through shuffles; every lane of the group returns the sum.
template <int G>
__device__ __forceinline__ double sor_row_sum(const double* x, const int* rcol, const double* rval, int len) {
    constexpr int kQ = 32 / G;
    const int lane = threadIdx.x & 31;
    const int glane = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    const int wlen = __reduce_max_sync(kFull, len);
    double s = 0.0;
    for (int base = 0; base < wlen; base += G * kQ) {
        double prod[kQ];
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            const int j = base + q * G + glane;
            prod[q] = j < len ? rval[j] * __ldcg(x + rcol[j]) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            if (base + q * G >= wlen) break;  // warp-uniform
#pragma unroll
            for (int i = 0; i < G; ++i) {
                const double t = __shfl_sync(kFull, prod[q], gbase + i);
                if (base + q * G + i < len) s = s + t;
            }
        }
    }
    return s;
}

template <int G, bool SMEM>
__global__ void __launch_bounds__(512) k_depth_sor(SorParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (failed(p.ctl)) return;  // set by an earlier kernel: the same for every CTA
    const int c = blockIdx.x, nc = gridDim.x;
    const int groups = blockDim.x / G;
    const int warp_first_group = (threadIdx.x >> 5) * (32 / G);
    const int my_group = (threadIdx.x & 31) / G;
    const int L = p.n_levels, D = p.stride;
    // shared-memory image: values [batch][nloc_max][max_row]; rhs, diagonal
    // and current x of the owned vertices [batch][nloc_max] (x is written
    // through to global memory for the other CTAs' gathers); columns
    // [nloc_max][max_row], vertex ids, row lengths, per-level owned ranges
    const long long nb = static_cast<long long>(p.batch) * p.nloc_max;
    double* sval = reinterpret_cast<double*>(smem_raw);
    double* srhs = sval + (SMEM ? nb * p.max_row : 0);
    double* sdiag = srhs + (SMEM ? nb : 0);
    double* sx = sdiag + (SMEM ? nb : 0);
    int* scol = reinterpret_cast<int*>(sx + (SMEM ? nb : 0));
    int* svid = scol + (SMEM ? p.nloc_max * p.max_row : 0);
    int* slen = svid + p.nloc_max;
    int* lbeg = slen + p.nloc_max;
    int* lend = lbeg + L;
    if (SMEM) {
        const int nloc = owned_below(p.n, c, nc);
        for (int i = threadIdx.x; i < nloc; i += blockDim.x) {
            const int v = p.order[c + i * nc];
            const long long row = 3LL * p.inc_off[v] + v;
            int len = 3 * (p.inc_off[v + 1] - p.inc_off[v]) + 1;
            if (len > p.max_row) {
                if (atomicCAS(&p.ctl->status, CSG_OK, CSG_ERR_ARG) == CSG_OK) p.ctl->where = -1;
                len = p.max_row;
            }
            svid[i] = v;
            slen[i] = len;
            for (int j = 0; j < len; ++j) scol[i * p.max_row + j] = p.col[row + j];
            for (int b = 0; b < p.batch; ++b) {
                const long long slot = static_cast<long long>(b) * p.nloc_max + i;
                for (int j = 0; j < len; ++j) sval[slot * p.max_row + j] = p.val[b * p.nnz + row + j];
                const long long at = static_cast<long long>(b) * p.n + v;
                srhs[slot] = p.rhs[at];
                sdiag[slot] = p.diag[at];
                sx[slot] = p.x[at];
            }
        }
        for (int l = threadIdx.x; l < L; l += blockDim.x) {
            lbeg[l] = owned_below(p.level_begin[l], c, nc);
            lend[l] = owned_below(p.level_end[l], c, nc);
        }
        __syncthreads();
    }
    unsigned int phase = 0;
    int barrier_id = 0;
    const int span = (p.sweeps - 1) * D;  // host guarantees span + L < 2^31
    const int nsteps = span + L;
    int r = 0;
    for (int t = 0; t < nsteps; ++t, r = (r + 1 == D) ? 0 : r + 1) {
        int lo = t - span;
        if (lo < r) lo = r;
        const int hi = t < L ? t : (L - 1) - ((L - 1 - r) % D + D) % D;
        if (hi >= lo) {
            const int i0 = SMEM ? lbeg[lo] : owned_below(p.level_begin[lo], c, nc);
            const int i1 = SMEM ? lend[hi] : owned_below(p.level_end[hi], c, nc);
            const int count = i1 - i0;
            for (int base = warp_first_group; base < count * p.batch; base += groups) {
                const int w = base + my_group;
                int b = 0, i = -1, v = 0, len = 0;
                long long slot = 0;
                const int* rcol = nullptr;
                const double* rval = nullptr;
                double rhs = 0.0, diag = 1.0;
                if (w < count * p.batch) {
                    b = w / count;
                    i = i0 + w % count;
                    slot = static_cast<long long>(b) * p.nloc_max + i;
                    if (SMEM) {
                        v = svid[i];
                        len = slen[i];
                        rcol = scol + i * p.max_row;
                        rval = sval + slot * p.max_row;
                        rhs = srhs[slot];
                        diag = sdiag[slot];
                    } else {
                        v = p.order[c + i * nc];
                        const long long row = 3LL * p.inc_off[v] + v;
                        len = 3 * (p.inc_off[v + 1] - p.inc_off[v]) + 1;
                        rcol = p.col + row;
                        rval = p.val + b * p.nnz + row;
                        rhs = p.rhs[static_cast<long long>(b) * p.n + v];
                        diag = p.diag[static_cast<long long>(b) * p.n + v];
                    }
                }
                const double sum = sor_row_sum<G>(p.x + static_cast<long long>(b) * p.n, rcol, rval, len);
                if (len > 0 && (threadIdx.x & (G - 1)) == 0) {
                    const long long at = static_cast<long long>(b) * p.n + v;
                    const double xv = SMEM ? sx[slot] : __ldcg(p.x + at);
                    const double nx = xv + p.relaxation * (rhs - sum) / diag;
                    if (SMEM) sx[slot] = nx;
                    __stcg(p.x + at, nx);
                }
            }
        }
        if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    }
}

// ---------------------------------------------------------------- SOR, dataflow form
//
// The sweeps without a grid barrier per step, as the Surf2Sphere dataflow
// kernels do it: x[b][v] is published as two versioned words (the low and the
// high 32 bits of the double, each with the number of sweeps completed).  In
// colour-major Gauss-Seidel order a neighbour u comes before v exactly when
// level(u) < level(v) (the schedule's potential grows along that order), so
// sweep s of v needs earlier neighbours at version s and later neighbours and
// v itself at version s - 1, and none can be further ahead.  A group polls the
// row's distinct columns (its ring), stages their x in shared memory, forms
// the row sum in entry order and publishes the update.

constexpr int kSRing = 16;  // the vertex and at most 15 distinct neighbours

__global__ void k_level_of(const int* __restrict__ order, const int* __restrict__ level_begin,
                           const int* __restrict__ level_end, int* __restrict__ level_of) {
    const int l = blockIdx.y;
    for (int pos = level_begin[l] + blockIdx.x * blockDim.x + threadIdx.x; pos < level_end[l];
         pos += gridDim.x * blockDim.x)
        level_of[order[pos]] = l;
}

__device__ __forceinline__ double words_value(unsigned long long lo, unsigned long long hi) {
    return __hiloint2double(static_cast<int>(static_cast<unsigned>(hi)), static_cast<int>(static_cast<unsigned>(lo)));
}

template <int G>
__device__ __forceinline__ bool sor_row_df(const SorParams& p, int b, int v, const int* ring, int nring,
                                           const unsigned char* code, const double* rval, int len, double rhs,
                                           double diag, unsigned int s, double* ringx) {
    constexpr int kQ = (kSRing + G - 1) / G;
    constexpr int kE = 32 / G;  // entries per lane and block of 32
    const int lane = threadIdx.x & 31;
    const int glane = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    const unsigned long long* pub = p.pub + 2LL * p.n * b;
    if (v < 0) {
        nring = 0;
        len = 0;
    }
    unsigned int polls = 0;
    unsigned long long start = 0;
    int who[kQ];
    unsigned int need[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        const int k = glane + q * G;
        who[q] = k < nring ? (ring[k] & 0x7fffffff) : -1;
        need[q] = (k < nring && (ring[k] < 0)) ? s : s - 1;  // sign bit: the neighbour comes first
    }
    while (true) {
        unsigned long long w[kQ][2];
#pragma unroll
        for (int q = 0; q < kQ; ++q)
            if (who[q] >= 0) {
                w[q][0] = csg::ld_word(pub + 2LL * who[q]);
                w[q][1] = csg::ld_word(pub + 2LL * who[q] + 1);
            }
        bool ok = true;
#pragma unroll
        for (int q = 0; q < kQ; ++q)
            if (who[q] >= 0) {
                ok = ok && csg::word_version(w[q][0]) == need[q] && csg::word_version(w[q][1]) == need[q];
                ringx[glane + q * G] = words_value(w[q][0], w[q][1]);
            }
        if (__all_sync(kFull, ok)) break;
        if (csg::warp_wait_expired(p.ctl, p.timeout_ns, polls, start)) return false;
    }
    __syncwarp();
    const int wlen = __reduce_max_sync(kFull, len);
    double sum = 0.0;
    for (int base = 0; base < wlen; base += G * kE) {
        double prod[kE];
#pragma unroll
        for (int q = 0; q < kE; ++q) {
            const int j = base + q * G + glane;
            prod[q] = j < len ? rval[j] * ringx[code[j]] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kE; ++q) {
            if (base + q * G >= wlen) break;  // warp-uniform
#pragma unroll
            for (int i = 0; i < G; ++i) {
                const double t = __shfl_sync(kFull, prod[q], gbase + i);
                if (base + q * G + i < len) sum = sum + t;
            }
        }
    }
    const double xv = v >= 0 ? ringx[0] : 0.0;
    __syncwarp();  // every lane is done with `ringx` before the next row overwrites it
    if (v >= 0 && glane < 2) {
        const double nx = xv + p.relaxation * (rhs - sum) / diag;
        const unsigned int half = glane == 0 ? static_cast<unsigned>(__double2loint(nx))
                                             : static_cast<unsigned>(__double2hiint(nx));
        csg::st_word(p.pub + 2LL * p.n * b + 2LL * v + glane, csg::make_word(__uint_as_float(half), s));
    }
    return true;
}

template <int G>
__global__ void __launch_bounds__(512) k_depth_sor_df(SorParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (failed(p.ctl)) return;  // set by an earlier kernel: the same for every CTA
    const int c = blockIdx.x, nc = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    const int groups = blockDim.x / G;
    const int warp_first_group = (threadIdx.x >> 5) * (32 / G);
    const int my_group = (threadIdx.x & 31) / G;
    const int L = p.n_levels, D = p.stride;
    // shared-memory image: per group kSRing staged x; values [batch][nloc][max_row];
    // rhs and diagonal [batch][nloc]; rings [nloc][kSRing] (sign bit: the neighbour
    // comes first); entry codes [nloc][max_row]; ids, ring sizes, row lengths,
    // levels; per-level owned ranges
    const long long nb = static_cast<long long>(p.batch) * p.nloc_max;
    double* ringx = reinterpret_cast<double*>(smem_raw) + (threadIdx.x / G) * kSRing;
    double* sval = reinterpret_cast<double*>(smem_raw) + (blockDim.x / G) * kSRing;
    double* srhs = sval + nb * p.max_row;
    double* sdiag = srhs + nb;
    int* sring = reinterpret_cast<int*>(sdiag + nb);
    int* svid = sring + p.nloc_max * kSRing;
    int* snring = svid + p.nloc_max;
    int* slen = snring + p.nloc_max;
    int* slev = slen + p.nloc_max;
    int* lbeg = slev + p.nloc_max;
    int* lend = lbeg + L;
    unsigned char* scode = reinterpret_cast<unsigned char*>(lend + L);
    const int nloc = owned_below(p.n, c, nc);
    for (int i = threadIdx.x; i < nloc; i += blockDim.x) {
        const int v = p.order[c + i * nc];
        const long long row = 3LL * p.inc_off[v] + v;
        int len = 3 * (p.inc_off[v + 1] - p.inc_off[v]) + 1;
        bool bad = len > p.max_row;
        if (bad) len = p.max_row;
        const int lv = p.level_of[v];
        int* ring = sring + i * kSRing;
        int nr = 1;
        ring[0] = v;
        for (int j = 0; j < len; ++j) {
            const int u = p.col[row + j];
            int at = 0;
            while (at < nr && (ring[at] & 0x7fffffff) != u) ++at;
            if (at == nr) {
                if (nr == kSRing) {
                    bad = true;
                    at = 0;
                } else {
                    ring[nr++] = p.level_of[u] < lv ? (u | static_cast<int>(0x80000000u)) : u;
                }
            }
            scode[static_cast<long long>(i) * p.max_row + j] = static_cast<unsigned char>(at);
        }
        if (bad && atomicCAS(&p.ctl->status, CSG_OK, CSG_ERR_ARG) == CSG_OK) p.ctl->where = -1;
        snring[i] = nr;
        svid[i] = v;
        slen[i] = len;
        slev[i] = lv;
        for (int b = 0; b < p.batch; ++b) {
            const long long slot = static_cast<long long>(b) * p.nloc_max + i;
            for (int j = 0; j < len; ++j) sval[slot * p.max_row + j] = p.val[b * p.nnz + row + j];
            const long long at = static_cast<long long>(b) * p.n + v;
            srhs[slot] = p.rhs[at];
            sdiag[slot] = p.diag[at];
        }
    }
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        lbeg[l] = owned_below(p.level_begin[l], c, nc);
        lend[l] = owned_below(p.level_end[l], c, nc);
    }
    for (long long q = tid; q < static_cast<long long>(p.batch) * p.n; q += nthreads) {
        const double x = p.x[q];
        csg::st_word(p.pub + 2 * q, csg::make_word(__uint_as_float(static_cast<unsigned>(__double2loint(x))), 0u));
        csg::st_word(p.pub + 2 * q + 1, csg::make_word(__uint_as_float(static_cast<unsigned>(__double2hiint(x))), 0u));
    }
    unsigned int phase = 0;
    int barrier_id = 0;
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    if (csg::ld_relaxed_gpu(&p.ctl->status) != CSG_OK) return;  // an oversized row: same answer in every CTA
    const int span = (p.sweeps - 1) * D;  // host guarantees span + L < 2^31
    const int nsteps = span + L;
    int r = 0, rot = 0;
    for (int t = 0; t < nsteps; ++t, r = (r + 1 == D) ? 0 : r + 1) {
        int lo = t - span;
        if (lo < r) lo = r;
        const int hi = t < L ? t : (L - 1) - ((L - 1 - r) % D + D) % D;
        if (hi < lo) continue;
        const int i0 = lbeg[lo], i1 = lend[hi];
        const int count = i1 - i0;
        for (int k0 = csg::dealt_first(rot, warp_first_group, groups); k0 < count * p.batch; k0 += groups) {
            const int w = k0 + my_group;
            int b = 0, i = 0, v = -1, nring = 0, len = 0;
            unsigned int sweep = 0;
            const int* ring = nullptr;
            const unsigned char* code = nullptr;
            const double* rval = nullptr;
            double rhs = 0.0, diag = 1.0;
            if (w >= 0 && w < count * p.batch) {
                b = w / count;
                i = i0 + w % count;
                const long long slot = static_cast<long long>(b) * p.nloc_max + i;
                v = svid[i];
                nring = snring[i];
                len = slen[i];
                ring = sring + i * kSRing;
                code = scode + static_cast<long long>(i) * p.max_row;
                rval = sval + slot * p.max_row;
                rhs = srhs[slot];
                diag = sdiag[slot];
                sweep = static_cast<unsigned int>(1 + (t - slev[i]) / D);
            }
            if (!sor_row_df<G>(p, b, v, ring, nring, code, rval, len, rhs, diag, sweep, ringx)) return;
        }
        rot = (rot + count * p.batch) % groups;
    }
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    for (long long q = tid; q < static_cast<long long>(p.batch) * p.n; q += nthreads)
        p.x[q] = words_value(csg::ld_word(p.pub + 2 * q), csg::ld_word(p.pub + 2 * q + 1));
}

// residual terms (rhs - A x)^2 per vertex (also the matrix-vector product of CG's start)
__global__ void k_depth_residual_terms(const int* inc_off, const int* col, const double* val, const double* rhs,
                                       const double* x, long long nnz, int n, int batch, double* terms,
                                       const csg::Control* ctl) {
    if (failed(ctl)) return;
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(n) * batch) return;
    const int b = static_cast<int>(i / n), v = static_cast<int>(i % n);
    const long long row = 3LL * inc_off[v] + v;
    const int len = 3 * (inc_off[v + 1] - inc_off[v]) + 1;
    const double* xb = x + static_cast<long long>(b) * n;
    const double* vb = val + b * nnz + row;
    double s = 0.0;
    for (int j = 0; j < len; ++j) s = s + vb[j] * xb[col[row + j]];
    const double r = rhs[i] - s;
    terms[i] = r * r;
}

__global__ void k_depth_residual_finish(const double* terms, int n, const double* rhs_norm, double* residual,
                                        int* iterations, int sweeps, double* runs_buf, const csg::Control* ctl) {
    if (failed(ctl)) return;
    const int b = blockIdx.x;
    const double* t = terms + static_cast<long long>(b) * n;
    double* buf = runs_buf + static_cast<long long>(b) * ((n + kRun - 1) / kRun + 1);
    const double s = cta_blocked_sum(n, [&](int i) { return t[i]; }, buf);
    if (threadIdx.x == 0) {
        residual[b] = sqrt(s) / rhs_norm[b];
        iterations[b] = sweeps;
    }
}

// ---------------------------------------------------------------- CG

struct CgParams {
    const int* inc_off;
    const int* col;
    const double* val;
    const double* diag;
    const double* rhs;
    const double* rhs_norm;
    double* x;
    double* r;
    double* z;
    double* pv;
    double* ap;
    double* terms;  // [batch][n]
    double* runs;   // [batch][runs]
    int* iterations;
    double* residual;
    csg::Control* ctl;
    long long nnz;
    int n, batch, max_iter;
    double tolerance;
    unsigned long long timeout_ns;
};

// Blocked sums of terms[b][0..n) for every surface: run sums by the whole
// grid, a grid barrier, then every CTA folds the runs the same way.
__device__ bool grid_blocked_sums(const CgParams& p, unsigned int& phase, int& barrier_id, double* out) {
    __shared__ double s_out[kMaxCgBatch];
    const int runs = (p.n + kRun - 1) / kRun;
    const long long total = static_cast<long long>(runs) * p.batch;
    const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (long long q = tid; q < total; q += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(q / runs), rr = static_cast<int>(q % runs);
        const double* t = p.terms + static_cast<long long>(b) * p.n;
        double s = 0.0;
        const int e = min(p.n, (rr + 1) * kRun);
        for (int i = rr * kRun; i < e; ++i) s = s + __ldcg(t + i);
        __stcg(p.runs + q, s);
    }
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return true;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int b = warp; b < p.batch; b += blockDim.x >> 5) {
        double acc = 0.0;
        for (int rr = lane; rr < runs; rr += 32) acc = acc + __ldcg(p.runs + static_cast<long long>(b) * runs + rr);
        for (int off = 16; off >= 1; off >>= 1) acc = acc + __shfl_down_sync(kFull, acc, off);
        if (lane == 0) s_out[b] = acc;
    }
    __syncthreads();
    for (int b = 0; b < p.batch; ++b) out[b] = s_out[b];
    __syncthreads();
    return false;
}

__device__ __forceinline__ double cg_row(const CgParams& p, int b, int v, const double* vec) {
    const long long row = 3LL * p.inc_off[v] + v;
    const int len = 3 * (p.inc_off[v + 1] - p.inc_off[v]) + 1;
    const double* vb = p.val + b * p.nnz + row;
    const double* xb = vec + static_cast<long long>(b) * p.n;
    double s = 0.0;
    for (int j = 0; j < len; ++j) s = s + vb[j] * __ldcg(xb + p.col[row + j]);
    return s;
}

__global__ void __launch_bounds__(512) k_depth_cg(CgParams p) {
    if (failed(p.ctl)) return;  // set by an earlier kernel: the same for every CTA
    unsigned int phase = 0;
    int barrier_id = 0;
    const long long total = static_cast<long long>(p.n) * p.batch;
    const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long nthreads = static_cast<long long>(gridDim.x) * blockDim.x;
    double rho[kMaxCgBatch], sums[kMaxCgBatch];
    bool done[kMaxCgBatch];
    // x = 0 (zeroed before the launch), r = rhs - A x
    for (long long i = tid; i < total; i += nthreads) {
        const int b = static_cast<int>(i / p.n), v = static_cast<int>(i % p.n);
        const double r = p.rhs[i] - cg_row(p, b, v, p.x);
        __stcg(p.r + i, r);
        __stcg(p.terms + i, r * r);
    }
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    if (grid_blocked_sums(p, phase, barrier_id, sums)) return;
    bool all_done = true;
    for (int b = 0; b < p.batch; ++b) {
        const double rel = sqrt(sums[b]) / p.rhs_norm[b];
        done[b] = rel <= p.tolerance;
        all_done = all_done && done[b];
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            p.residual[b] = rel;
            p.iterations[b] = 0;
        }
    }
    if (all_done) return;
    for (long long i = tid; i < total; i += nthreads) {
        const double z = __ldcg(p.r + i) / p.diag[i];
        __stcg(p.z + i, z);
        __stcg(p.pv + i, z);
        __stcg(p.terms + i, __ldcg(p.r + i) * z);
    }
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    if (grid_blocked_sums(p, phase, barrier_id, rho)) return;
    for (int it = 1; it <= p.max_iter; ++it) {
        // ap = A p, terms = p ap (surfaces already converged keep their state)
        for (long long i = tid; i < total; i += nthreads) {
            const int b = static_cast<int>(i / p.n), v = static_cast<int>(i % p.n);
            if (done[b]) continue;
            const double ap = cg_row(p, b, v, p.pv);
            __stcg(p.ap + i, ap);
            __stcg(p.terms + i, __ldcg(p.pv + i) * ap);
        }
        if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
        if (grid_blocked_sums(p, phase, barrier_id, sums)) return;
        for (long long i = tid; i < total; i += nthreads) {
            const int b = static_cast<int>(i / p.n);
            if (done[b]) continue;
            const double step = rho[b] / sums[b];
            __stcg(p.x + i, __ldcg(p.x + i) + step * __ldcg(p.pv + i));
            const double r = __ldcg(p.r + i) - step * __ldcg(p.ap + i);
            __stcg(p.r + i, r);
            __stcg(p.terms + i, r * r);
        }
        if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
        if (grid_blocked_sums(p, phase, barrier_id, sums)) return;
        bool stopped[kMaxCgBatch];
        all_done = true;
        for (int b = 0; b < p.batch; ++b) {
            stopped[b] = false;
            if (done[b]) continue;
            const double rel = sqrt(sums[b]) / p.rhs_norm[b];
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                p.residual[b] = rel;
                p.iterations[b] = it;
            }
            if (rel <= p.tolerance) stopped[b] = true;
            all_done = all_done && stopped[b];
        }
        if (all_done) return;
        for (long long i = tid; i < total; i += nthreads) {
            const int b = static_cast<int>(i / p.n);
            if (done[b] || stopped[b]) continue;
            const double z = __ldcg(p.r + i) / p.diag[i];
            __stcg(p.z + i, z);
            __stcg(p.terms + i, __ldcg(p.r + i) * z);
        }
        if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
        if (grid_blocked_sums(p, phase, barrier_id, sums)) return;
        for (long long i = tid; i < total; i += nthreads) {
            const int b = static_cast<int>(i / p.n);
            if (done[b] || stopped[b]) continue;
            const double beta = sums[b] / rho[b];
            __stcg(p.pv + i, __ldcg(p.z + i) + beta * __ldcg(p.pv + i));
        }
        for (int b = 0; b < p.batch; ++b) {
            if (done[b] || stopped[b]) {
                done[b] = true;
                continue;
            }
            rho[b] = sums[b];
        }
        if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    }
}

// ---------------------------------------------------------------- host side

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct Layout {
    size_t ctl, rec, col, val, areas, diag, mc, rhs, rhs_norm, runs, terms, r, z, pv, ap, pub, level_of, total;
};

Layout layout(int n, int nf, int batch, long long nnz) {
    Layout L{};
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t here = at;
        at += align256(bytes);
        return here;
    };
    const size_t nb = static_cast<size_t>(n) * batch;
    L.ctl = take(sizeof(csg::Control));
    L.rec = take(sizeof(double) * kRec * static_cast<size_t>(nf) * batch);
    L.col = take(sizeof(int) * static_cast<size_t>(nnz));
    L.val = take(sizeof(double) * static_cast<size_t>(nnz) * batch);
    L.areas = take(8 * nb);
    L.diag = take(8 * nb);
    L.mc = take(8 * nb);
    L.rhs = take(8 * nb);
    L.rhs_norm = take(8 * static_cast<size_t>(batch));
    L.runs = take(8 * (static_cast<size_t>(n) / kRun + 2) * batch);
    L.terms = take(8 * nb);
    L.r = take(8 * nb);
    L.z = take(8 * nb);
    L.pv = take(8 * nb);
    L.ap = take(8 * nb);
    L.pub = take(16 * nb);
    L.level_of = take(4 * static_cast<size_t>(n));
    L.total = at;
    return L;
}

inline unsigned blocks(long long n, int threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

constexpr size_t kMaxRowSmem = 200 * 1024;

template <int G, bool SMEM>
int launch_sor(const SorParams& params, int n_ctas, int threads, size_t smem, cudaStream_t s) {
    auto kernel = k_depth_sor<G, SMEM>;
    int device = 0, sms = 0, per_sm = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CSG_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1 || n_ctas > per_sm * sms)
        return csg::fail(CSG_ERR_LAUNCH, "depth SOR: %d CTAs x %d threads (%zu B smem) cannot be co-resident", n_ctas,
                         threads, smem);
    SorParams p = params;
    void* args[] = {&p};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(n_ctas), dim3(threads), args,
                                               smem, s));
    csg::note_launch();
    return CSG_OK;
}

template <int G>
int launch_sor_df(const SorParams& params, int n_ctas, int threads, size_t smem, cudaStream_t s) {
    auto kernel = k_depth_sor_df<G>;
    int device = 0, sms = 0, per_sm = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CSG_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1 || n_ctas > per_sm * sms)
        return csg::fail(CSG_ERR_LAUNCH, "depth SOR: %d CTAs x %d threads (%zu B smem) cannot be co-resident", n_ctas,
                         threads, smem);
    SorParams p = params;
    void* args[] = {&p};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(n_ctas), dim3(threads), args,
                                               smem, s));
    csg::note_launch();
    return CSG_OK;
}

template <int G>
int dispatch_sor(SorParams p, int n_ctas, int threads, cudaStream_t s) {
    p.nloc_max = (p.n + n_ctas - 1) / n_ctas;
    // dataflow form: a row's distinct columns (at most 2 max_incidences + 1) fit the ring
    if (p.pub && p.max_row > 0 && p.max_row <= 255 && 2 * ((p.max_row - 1) / 3) + 1 <= kSRing) {
        const long long nb = static_cast<long long>(p.batch) * p.nloc_max;
        const size_t smem = sizeof(double) * (static_cast<size_t>(threads / G) * kSRing + nb * (p.max_row + 2)) +
                            sizeof(int) * (static_cast<size_t>(p.nloc_max) * (kSRing + 5) + 2 * static_cast<size_t>(p.n_levels)) +
                            static_cast<size_t>(p.nloc_max) * p.max_row;
        if (smem <= kMaxRowSmem) return launch_sor_df<G>(p, n_ctas, threads, smem, s);
    }
    const size_t ints = static_cast<size_t>(p.nloc_max) * (p.max_row + 2) + 2 * static_cast<size_t>(p.n_levels);
    const size_t smem = sizeof(double) * static_cast<size_t>(p.batch) * p.nloc_max * (p.max_row + 3) + sizeof(int) * ints;
    if (p.max_row > 0 && smem <= kMaxRowSmem) return launch_sor<G, true>(p, n_ctas, threads, smem, s);
    p.max_row = 0;
    return launch_sor<G, false>(p, n_ctas, threads, 0, s);
}

}  // namespace

extern "C" {

size_t csg_depth_scratch_bytes(int n_vertices, int n_faces, int batch) {
    if (n_vertices < 3 || n_faces < 1 || batch < 1) return 0;
    return layout(n_vertices, n_faces, batch, 9LL * n_faces + n_vertices).total;
}

int csg_depth_potential(const float* geometry, int batch, int n, const int32_t* faces, int nf, const int32_t* inc_off,
                        const int32_t* inc, int max_incidences, double alpha, int solver,
                        int max_iter, double tolerance, double relaxation, const int32_t* order,
                        const int32_t* level_begin, const int32_t* level_end, int n_levels, int level_stride,
                        double* values, int32_t* iterations, double* residual, double* normals, double* areas,
                        void* scratch, size_t scratch_bytes, int n_ctas, int threads_per_cta, int lanes_per_row,
                        double timeout_s, csg_stream_t stream) {
    if (!geometry || batch < 1 || n < 3 || !faces || nf < 1 || !inc_off || !inc ||
        max_incidences < 1 || !(alpha != 0.0) || !std::isfinite(alpha) || max_iter < 0 || !values || !iterations ||
        !residual || !scratch)
        return csg::fail(CSG_ERR_ARG, "depth potential: bad arguments");
    if (solver != CSG_DEPTH_SOR && solver != CSG_DEPTH_PCG)
        return csg::fail(CSG_ERR_ARG, "depth potential: solver must be CSG_DEPTH_SOR or CSG_DEPTH_PCG");
    if (solver == CSG_DEPTH_SOR &&
        (!order || !level_begin || !level_end || n_levels < 1 || n_levels > 65535 || level_stride < 1))
        return csg::fail(CSG_ERR_ARG, "depth potential: the SOR solver needs the colour-major wavefront schedule");
    if (solver == CSG_DEPTH_PCG && (max_iter < 1 || batch > kMaxCgBatch))
        return csg::fail(CSG_ERR_ARG, "depth potential: CG needs max_iter >= 1 and batch <= %d", kMaxCgBatch);
    if (solver == CSG_DEPTH_SOR &&
        static_cast<double>(max_iter > 0 ? max_iter - 1 : 0) * level_stride + n_levels >= 2147483647.0)
        return csg::fail(CSG_ERR_ARG, "depth potential: schedule too long");
    if (threads_per_cta <= 0) threads_per_cta = 512;
    if (threads_per_cta % 32 || threads_per_cta > 512) return csg::fail(CSG_ERR_ARG, "depth potential: threads 32..512, x32");
    if (lanes_per_row <= 0) lanes_per_row = 4;
    if (lanes_per_row != 4 && lanes_per_row != 8 && lanes_per_row != 16)
        return csg::fail(CSG_ERR_ARG, "depth potential: lanes_per_row must be 4, 8 or 16");
    if (timeout_s <= 0.0) timeout_s = 2.0;
    const long long nnz = 9LL * nf + n;  // 3 entries per incidence, 3 incidences per face, one alpha entry per row
    const Layout L = layout(n, nf, batch, nnz);
    if (scratch_bytes < L.total) return csg::fail(CSG_ERR_ARG, "depth potential: scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(scratch);
    auto* ctl = reinterpret_cast<csg::Control*>(base + L.ctl);
    SetupParams sp{};
    sp.geom = geometry;
    sp.faces = faces;
    sp.inc_off = inc_off;
    sp.inc = inc;
    sp.n = n;
    sp.nf = nf;
    sp.batch = batch;
    sp.alpha = alpha;
    sp.rec = reinterpret_cast<double*>(base + L.rec);
    sp.col = reinterpret_cast<int*>(base + L.col);
    sp.val = reinterpret_cast<double*>(base + L.val);
    sp.areas = areas ? areas : reinterpret_cast<double*>(base + L.areas);
    sp.diag = reinterpret_cast<double*>(base + L.diag);
    sp.mc = reinterpret_cast<double*>(base + L.mc);
    sp.rhs = reinterpret_cast<double*>(base + L.rhs);
    sp.rhs_norm = reinterpret_cast<double*>(base + L.rhs_norm);
    sp.normals = normals;
    sp.ctl = ctl;
    sp.nnz = nnz;
    double* runs = reinterpret_cast<double*>(base + L.runs);
    CSG_CUDA_CHECK(cudaMemsetAsync(ctl, 0, sizeof(csg::Control), s));
    (csg::note_launch(), k_depth_faces<<<blocks(static_cast<long long>(nf) * batch, kThreads), kThreads, 0, s>>>(sp));
    (csg::note_launch(), k_depth_vertices<<<blocks(static_cast<long long>(n) * batch, kThreads), kThreads, 0, s>>>(sp));
    (csg::note_launch(), k_depth_rhs<<<batch, 1024, 0, s>>>(sp, runs));
    CSG_CUDA_CHECK(cudaGetLastError());
    int device = 0, sms = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (n_ctas <= 0) n_ctas = sms;
    const unsigned long long timeout_ns = static_cast<unsigned long long>(timeout_s * 1e9);
    if (solver == CSG_DEPTH_SOR) {
        CSG_CUDA_CHECK(cudaMemsetAsync(values, 0, sizeof(double) * static_cast<size_t>(n) * batch, s));
        if (max_iter > 0) {
            SorParams p{};
            p.inc_off = inc_off;
            p.col = sp.col;
            p.val = sp.val;
            p.diag = sp.diag;
            p.rhs = sp.rhs;
            p.x = values;
            p.order = order;
            p.level_begin = level_begin;
            p.level_end = level_end;
            p.ctl = ctl;
            p.nnz = nnz;
            p.n = n;
            p.batch = batch;
            p.n_levels = n_levels;
            p.stride = level_stride;
            p.sweeps = max_iter;
            p.max_row = 3 * max_incidences + 1;
            p.relaxation = relaxation;
            p.timeout_ns = timeout_ns;
            p.pub = reinterpret_cast<unsigned long long*>(base + L.pub);
            p.level_of = reinterpret_cast<int*>(base + L.level_of);
            (csg::note_launch(), k_level_of<<<dim3(blocks(n, kThreads) > 64 ? 64 : blocks(n, kThreads), n_levels),
                                              kThreads, 0, s>>>(order, level_begin, level_end, p.level_of));
            int rc;
            switch (lanes_per_row) {
                case 8: rc = dispatch_sor<8>(p, n_ctas, threads_per_cta, s); break;
                case 16: rc = dispatch_sor<16>(p, n_ctas, threads_per_cta, s); break;
                default: rc = dispatch_sor<4>(p, n_ctas, threads_per_cta, s); break;
            }
            if (rc) return rc;
        }
        double* terms = reinterpret_cast<double*>(base + L.terms);
        (csg::note_launch(), k_depth_residual_terms<<<blocks(static_cast<long long>(n) * batch, kThreads), kThreads, 0, s>>>(
            inc_off, sp.col, sp.val, sp.rhs, values, nnz, n, batch, terms, ctl));
        (csg::note_launch(), k_depth_residual_finish<<<batch, 1024, 0, s>>>(terms, n, sp.rhs_norm, residual, iterations,
                                                                           max_iter, runs, ctl));
    } else {
        CSG_CUDA_CHECK(cudaMemsetAsync(values, 0, sizeof(double) * static_cast<size_t>(n) * batch, s));
        CgParams p{};
        p.inc_off = inc_off;
        p.col = sp.col;
        p.val = sp.val;
        p.diag = sp.diag;
        p.rhs = sp.rhs;
        p.rhs_norm = sp.rhs_norm;
        p.x = values;
        p.r = reinterpret_cast<double*>(base + L.r);
        p.z = reinterpret_cast<double*>(base + L.z);
        p.pv = reinterpret_cast<double*>(base + L.pv);
        p.ap = reinterpret_cast<double*>(base + L.ap);
        p.terms = reinterpret_cast<double*>(base + L.terms);
        p.runs = runs;
        p.iterations = iterations;
        p.residual = residual;
        p.ctl = ctl;
        p.nnz = nnz;
        p.n = n;
        p.batch = batch;
        p.max_iter = max_iter;
        p.tolerance = tolerance;
        p.timeout_ns = timeout_ns;
        auto kernel = k_depth_cg;
        int per_sm = 0;
        CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads_per_cta, 0));
        if (per_sm < 1 || n_ctas > per_sm * sms)
            return csg::fail(CSG_ERR_LAUNCH, "depth CG: %d CTAs x %d threads cannot be co-resident", n_ctas,
                             threads_per_cta);
        void* args[] = {&p};
        CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(n_ctas),
                                                   dim3(threads_per_cta), args, 0, s));
        csg::note_launch();
    }
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

}  // extern "C"
