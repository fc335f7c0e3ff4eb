// CAT_Surf2Sphere stages 1-5 (low_smooth, inflate, very_inflate, high_smooth,
// ellipsoid) on sm_100a.
//
// Semantics follow the reference's description of the upstream stages
// (src/cat_surface_gpu/surf2sphere.py:283-397, 474-862): per stage, keep the
// input as the reference geometry, centre on the vertex mean, then per cycle
// `iterations - 1` distance-smoothing passes, the inflation scale, the
// distortion selection and `finger_iterations - 1` passes over the selected
// vertices.  The passes are Gauss-Seidel in vertex index order -- the order
// the upstream binary uses (the reference's Triton path colours instead) --
// so they run as persistent cooperative wavefront kernels with the same
// schedule as the area-smoothing sweeps (vertex v of pass s at step
// s * D + level(v); the 1-ring is the dependency set of both).  The inflation
// is a pointwise pass of the same wavefront.  The global steps (centre,
// extents, face/vertex areas, the distortion selection) are plain kernels
// between launches: 19 wavefront launches for stages 1-5.
//
// Arithmetic: float32 positions, float64 arithmetic (one rounding per
// operation, --fmad=false).  Sums over all vertices or faces are blocked:
// sequential within runs of kBlockSum elements, then sequential over the
// runs, so results do not depend on the launch shape.
#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "common.cuh"
#include "errors.h"

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBlockSum = 256;
constexpr int kThreads = 256;

struct StageSpec {
    int cycles;
    double strength;
    int iterations;
    double inflation;
    double threshold;
    double finger_strength;
    int finger_iterations;
};

// surf2sphere.py:758-814
constexpr StageSpec kStages[5] = {
    {1, 0.2, 50, 1.0, 3.0, 1.0, 0},  {2, 1.0, 30, 1.4, 3.0, 1.0, 30}, {4, 1.0, 30, 1.1, 3.0, 1.0, 0},
    {6, 1.0, 60, 1.6, 3.0, 1.0, 60}, {6, 1.0, 50, 1.4, 4.0, 1.0, 60},
};

// Stage statistics kept on the device: mean[3], lo[3], hi[3], extent[3],
// reference surface, current surface.
struct Stats {
    double mean[3];
    double lo[3];
    double hi[3];
    double extent[3];
    double ref_surface;
    double cur_surface;
};

__device__ __forceinline__ float4 ld4(const float4* p, int v) { return __ldcg(p + v); }

// ---------------------------------------------------------------- passes

// A launch runs a list of segments back to back: a run of smoothing passes
// (over every vertex or over the selected ones) or one inflation pass.  The
// inflation scale is pointwise with stage-fixed statistics, so it is a pass of
// the same wavefront: vertex v is scaled after its own last smoothing pass and
// before any neighbour's next pass reads it, which is the order a separate
// kernel between two launches gives, without the pipeline drain in between.
enum SegmentKind : int { kSmoothAll = 0, kSmoothSelected = 1, kInflate = 2 };
constexpr int kMaxSegments = 8;

struct Segment {
    int first_pass;  // passes of earlier segments
    int kind;
    double value;  // smoothing strength, or the inflation's delta
};

struct PassParams {
    float4* work;
    unsigned long long* pub;  // dataflow form: 4 versioned words per vertex
    const int* nb_off;
    const int* nb;
    const unsigned char* selected;
    const Stats* st;
    const int* order;
    const int* level_begin;
    const int* level_end;
    csg::Control* ctl;
    int n;
    int n_levels;
    int stride;
    int passes;
    int n_segments;
    int max_degree;  // largest 1-ring (shared-memory variant)
    int nloc_max;    // most vertices one CTA owns (shared-memory variant)
    Segment seg[kMaxSegments];
    unsigned long long timeout_ns;
};

__device__ __forceinline__ void inflate_vertex(float4* work, int v, const Stats* st, double delta) {
    const float4 q = ld4(work, v);
    const double x = __ddiv_rn(q.x, st->extent[0]), y = __ddiv_rn(q.y, st->extent[1]), z = __ddiv_rn(q.z, st->extent[2]);
    const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    const double scale = __dadd_rn(1.0, __dmul_rn(delta, __dsub_rn(1.0, r)));
    __stcg(work + v, make_float4(__double2float_rn(__dmul_rn(q.x, scale)), __double2float_rn(__dmul_rn(q.y, scale)),
                                 __double2float_rn(__dmul_rn(q.z, scale)), 0.0f));
}

// One vertex of one pass of segment `sg` by a group of G lanes: lane j
// computes neighbour slots j, j + G, ... (L1 distance d, d q when d > 0), the
// terms are staged in shared memory and lanes 0..2 sum them in slot order
// (total and one coordinate each) and form that coordinate; lane 0 stores.
// An inflation segment scales the vertex by lane 0.  Groups of one warp may be
// in different segments; every lane takes the warp-wide steps.
template <int G>
__device__ __forceinline__ void smooth_vertex(const PassParams& p, int v, const int* ring, int deg, int sg,
                                              double (*stage)[32]) {
    const int lane = threadIdx.x & 31;
    const int glane = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    const int kind = p.seg[sg].kind;
    const double strength = p.seg[sg].value;
    bool active = v >= 0 && kind != kInflate && deg > 1 && (kind == kSmoothAll || p.selected[v]);
    if (!active) deg = 0;
    const int wdeg = __reduce_max_sync(kFull, deg);
    double o[3] = {0.0, 0.0, 0.0};
    if (active) {
        const float4 q = ld4(p.work, v);
        o[0] = q.x;
        o[1] = q.y;
        o[2] = q.z;
    }
    double total = 0.0, wsum = 0.0;
    const int comp = glane < 3 ? glane : 0;
    for (int c0 = 0; c0 < wdeg; c0 += G) {
        const int j = c0 + glane;
        double d = 0.0, dx = 0.0, dy = 0.0, dz = 0.0;
        if (j < deg) {
            const float4 q = ld4(p.work, ring[j]);
            const double qx = q.x, qy = q.y, qz = q.z;
            d = __dadd_rn(__dadd_rn(fabs(__dsub_rn(qx, o[0])), fabs(__dsub_rn(qy, o[1]))), fabs(__dsub_rn(qz, o[2])));
            if (d > 0.0) {
                dx = __dmul_rn(d, qx);
                dy = __dmul_rn(d, qy);
                dz = __dmul_rn(d, qz);
            }
        }
        stage[0][lane] = d;
        stage[1][lane] = dx;
        stage[2][lane] = dy;
        stage[3][lane] = dz;
        __syncwarp();
        if (glane < 3) {
            const int m = min(G, deg - c0);
#pragma unroll
            for (int q = 0; q < G; ++q) {
                if (q < m) {
                    total = __dadd_rn(total, stage[0][gbase + q]);
                    // the reference adds d q only for d > 0; the staged term is 0 otherwise
                    if (stage[0][gbase + q] > 0.0) wsum = __dadd_rn(wsum, stage[1 + comp][gbase + q]);
                }
            }
        }
        __syncwarp();
    }
    const double inv = 1.0 - strength;
    float c = 0.0f;
    if (active && glane < 3) {
        const double keep = __dmul_rn(o[comp], inv);
        c = __double2float_rn(total > 0.0 ? __dadd_rn(keep, __dmul_rn(__ddiv_rn(wsum, total), strength)) : keep);
    }
    const float cy = __shfl_sync(kFull, c, gbase + 1);
    const float cz = __shfl_sync(kFull, c, gbase + 2);
    if (active && glane == 0) __stcg(p.work + v, make_float4(c, cy, cz, 0.0f));
    if (kind == kInflate && v >= 0 && glane == 0) inflate_vertex(p.work, v, p.st, strength);
}

__device__ __forceinline__ int owned_below(int bound, int c, int nc) { return bound > c ? (bound - c + nc - 1) / nc : 0; }

// `passes` passes (the segments' runs back to back) as one wavefront (see
// the file comment).  CTA c owns order positions c, c + nc, ...  With SMEM the
// CTA first copies its vertices' ids and 1-rings and its per-level owned
// ranges into shared memory, so a step's only global loads are the positions.
template <int G, bool SMEM>
__global__ void __launch_bounds__(512) smooth_passes_kernel(PassParams p) {
    extern __shared__ int smem[];
    __shared__ double stage_all[512 / 32][4][32];
    double (*stage)[32] = stage_all[threadIdx.x >> 5];
    const int c = blockIdx.x, nc = gridDim.x;
    const int groups = blockDim.x / G;
    const int warp_first_group = (threadIdx.x >> 5) * (32 / G);
    const int my_group = (threadIdx.x & 31) / G;
    const int L = p.n_levels, D = p.stride;
    // shared-memory image: rings [nloc_max][max_degree], ids, degrees, and the
    // owned index range of every level
    int* lring = smem;
    int* lvid = lring + (SMEM ? p.nloc_max * p.max_degree : 0);
    int* ldeg = lvid + p.nloc_max;
    int* lbeg = ldeg + p.nloc_max;
    int* lend = lbeg + L;
    if (SMEM) {
        const int nloc = owned_below(p.n, c, nc);
        for (int i = threadIdx.x; i < nloc; i += blockDim.x) {
            const int v = __ldg(p.order + c + i * nc);
            const int b = __ldg(p.nb_off + v);
            int d = __ldg(p.nb_off + v + 1) - b;
            if (d > p.max_degree) {
                // a ring longer than the caller's max_degree: report it and
                // keep the copy inside the image
                if (atomicCAS(&p.ctl->status, CSG_OK, CSG_ERR_ARG) == CSG_OK) p.ctl->where = -1;
                d = p.max_degree;
            }
            lvid[i] = v;
            ldeg[i] = d;
            for (int j = 0; j < d; ++j) lring[i * p.max_degree + j] = __ldg(p.nb + b + j);
        }
        for (int l = threadIdx.x; l < L; l += blockDim.x) {
            lbeg[l] = owned_below(__ldg(p.level_begin + l), c, nc);
            lend[l] = owned_below(__ldg(p.level_end + l), c, nc);
        }
        __syncthreads();
    }
    unsigned int phase = 0;
    int barrier_id = 0;
    const int span = (p.passes - 1) * D;  // host guarantees span + L < 2^31
    const int nsteps = span + L;
    int r = 0;
    for (int t = 0; t < nsteps; ++t, r = (r + 1 == D) ? 0 : r + 1) {
        int lo = t - span;
        if (lo < r) lo = r;
        const int hi = t < L ? t : (L - 1) - ((L - 1 - r) % D + D) % D;
        if (hi >= lo) {
            const int i0 = SMEM ? lbeg[lo] : owned_below(__ldg(p.level_begin + lo), c, nc);
            const int i1 = SMEM ? lend[hi] : owned_below(__ldg(p.level_end + hi), c, nc);
            // Vertex v is in pass (t - level(v)) / D, so it has reached segment k
            // when level(v) <= t - first_pass_k * D; the range is sorted by
            // level, so that is every owned index below ib[k].
            int ib[kMaxSegments];
#pragma unroll
            for (int k = 1; k < kMaxSegments; ++k) {
                ib[k] = 0;
                if (k < p.n_segments) {
                    const int m = t - p.seg[k].first_pass * D;
                    ib[k] = m < lo ? i0
                                   : (m >= hi ? i1 : (SMEM ? lend[m] : owned_below(__ldg(p.level_end + m), c, nc)));
                }
            }
            for (int base = i0 + warp_first_group; base < i1; base += groups) {
                const int i = base + my_group;
                int v = -1, deg = 0;
                const int* ring = nullptr;
                if (i < i1) {
                    if (SMEM) {
                        v = lvid[i];
                        deg = ldeg[i];
                        ring = lring + i * p.max_degree;
                    } else {
                        v = __ldg(p.order + c + i * nc);
                        const int b = __ldg(p.nb_off + v);
                        deg = __ldg(p.nb_off + v + 1) - b;
                        ring = p.nb + b;
                    }
                }
                int sg = 0;
#pragma unroll
                for (int k = 1; k < kMaxSegments; ++k) sg += i < ib[k];
                smooth_vertex<G>(p, v, ring, deg, sg, stage);
            }
        }
        if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    }
}

// ---------------------------------------------------------------- dataflow form
//
// The same passes without a grid barrier per wavefront step: each coordinate
// is published as a versioned word (csg::make_word; version = passes the
// vertex has completed in this launch).  Pass k of vertex v needs its
// lower-index neighbours at version k + 1, its higher-index neighbours and
// itself at version k, and none of them can be further ahead (a neighbour's
// next pass needs v's pass k), so the words that show those versions hold
// exactly the values the sequential order reads.  A group polls the ring (v
// and its 1-ring, one round trip per poll), stages the positions in shared
// memory and applies the segment's update; every vertex publishes every pass
// (unchanged when it does not move).  Grid barriers remain at the start (the
// words are written from `work`) and at the end (`work` is written back).

constexpr int kPRing = 17;  // the vertex and at most 16 neighbours

template <int G>
__device__ __forceinline__ bool pass_vertex_df(const PassParams& p, int v, const int* ring, int nring, int sg,
                                               unsigned int pass, double (*stage)[32], float3* pos) {
    constexpr int kQ = (kPRing + G - 1) / G;
    const int lane = threadIdx.x & 31;
    const int glane = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    const int kind = p.seg[sg].kind;
    const double strength = p.seg[sg].value;
    if (v < 0) nring = 0;
    unsigned int polls = 0;
    unsigned long long start = 0;
    int who[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        const int k = glane + q * G;
        who[q] = k < nring ? ring[k] : -1;
    }
    while (true) {
        unsigned long long w[kQ][3];
#pragma unroll
        for (int q = 0; q < kQ; ++q)
            if (who[q] >= 0)
#pragma unroll
                for (int k = 0; k < 3; ++k) w[q][k] = csg::ld_word(p.pub + 4LL * who[q] + k);
        bool ok = true;
#pragma unroll
        for (int q = 0; q < kQ; ++q)
            if (who[q] >= 0) {
                const unsigned int need = who[q] < v ? pass + 1 : pass;  // the vertex itself: pass
                ok = ok && csg::word_version(w[q][0]) == need && csg::word_version(w[q][1]) == need &&
                     csg::word_version(w[q][2]) == need;
                pos[glane + q * G] = make_float3(csg::word_value(w[q][0]), csg::word_value(w[q][1]),
                                                 csg::word_value(w[q][2]));
            }
        if (__all_sync(kFull, ok)) break;
        if (csg::warp_wait_expired(p.ctl, p.timeout_ns, polls, start)) return false;
    }
    __syncwarp();
    int deg = nring > 0 ? nring - 1 : 0;
    const bool active = v >= 0 && kind != kInflate && deg > 1 && (kind == kSmoothAll || p.selected[v]);
    if (!active) deg = 0;
    const int wdeg = __reduce_max_sync(kFull, deg);
    double o[3] = {0.0, 0.0, 0.0};
    if (v >= 0) {
        o[0] = pos[0].x;
        o[1] = pos[0].y;
        o[2] = pos[0].z;
    }
    double total = 0.0, wsum = 0.0;
    const int comp = glane < 3 ? glane : 0;
    for (int c0 = 0; c0 < wdeg; c0 += G) {
        const int j = c0 + glane;
        double d = 0.0, dx = 0.0, dy = 0.0, dz = 0.0;
        if (j < deg) {
            const float3 q = pos[1 + j];
            const double qx = q.x, qy = q.y, qz = q.z;
            d = __dadd_rn(__dadd_rn(fabs(__dsub_rn(qx, o[0])), fabs(__dsub_rn(qy, o[1]))), fabs(__dsub_rn(qz, o[2])));
            if (d > 0.0) {
                dx = __dmul_rn(d, qx);
                dy = __dmul_rn(d, qy);
                dz = __dmul_rn(d, qz);
            }
        }
        stage[0][lane] = d;
        stage[1][lane] = dx;
        stage[2][lane] = dy;
        stage[3][lane] = dz;
        __syncwarp();
        if (glane < 3) {
            const int m = min(G, deg - c0);
#pragma unroll
            for (int q = 0; q < G; ++q) {
                if (q < m) {
                    total = __dadd_rn(total, stage[0][gbase + q]);
                    // the reference adds d q only for d > 0; the staged term is 0 otherwise
                    if (stage[0][gbase + q] > 0.0) wsum = __dadd_rn(wsum, stage[1 + comp][gbase + q]);
                }
            }
        }
        __syncwarp();
    }
    float value = 0.0f;
    if (v >= 0 && glane < 3) {
        if (active) {
            const double keep = __dmul_rn(o[comp], 1.0 - strength);
            value = __double2float_rn(total > 0.0 ? __dadd_rn(keep, __dmul_rn(__ddiv_rn(wsum, total), strength)) : keep);
        } else if (kind == kInflate) {
            const Stats* st = p.st;
            const double x = __ddiv_rn(o[0], st->extent[0]), y = __ddiv_rn(o[1], st->extent[1]),
                         z = __ddiv_rn(o[2], st->extent[2]);
            const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
            const double scale = __dadd_rn(1.0, __dmul_rn(strength, __dsub_rn(1.0, r)));
            value = __double2float_rn(__dmul_rn(o[comp], scale));
        } else {
            value = static_cast<float>(o[comp]);
        }
    }
    __syncwarp();  // every lane is done with `pos` before the next update overwrites it
    if (v >= 0 && glane < 3) csg::st_word(p.pub + 4LL * v + glane, csg::make_word(value, pass + 1));
    return true;
}

template <int G>
__global__ void __launch_bounds__(512) smooth_passes_df(PassParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double stage_all[512 / 32][4][32];
    double (*stage)[32] = stage_all[threadIdx.x >> 5];
    const int c = blockIdx.x, nc = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    const int groups = blockDim.x / G;
    const int warp_first_group = (threadIdx.x >> 5) * (32 / G);
    const int my_group = (threadIdx.x & 31) / G;
    const int L = p.n_levels, D = p.stride;
    // shared-memory image: per warp, kPRing staged positions per group; per
    // owned vertex its ring (itself, then its 1-ring), ring size, id and level;
    // per level the owned range
    float3* pos = reinterpret_cast<float3*>(smem_raw) + ((threadIdx.x >> 5) * (32 / G) + my_group) * kPRing;
    int* lring = reinterpret_cast<int*>(reinterpret_cast<float3*>(smem_raw) + (blockDim.x / G) * kPRing);
    int* lnring = lring + p.nloc_max * kPRing;
    int* lvid = lnring + p.nloc_max;
    int* llev = lvid + p.nloc_max;
    int* lbeg = llev + p.nloc_max;
    int* lend = lbeg + L;
    const int nloc = owned_below(p.n, c, nc);
    for (int i = threadIdx.x; i < nloc; i += blockDim.x) {
        const int v = __ldg(p.order + c + i * nc);
        const int b = __ldg(p.nb_off + v);
        int d = __ldg(p.nb_off + v + 1) - b;
        if (d > p.max_degree || d + 1 > kPRing) {  // a ring longer than the caller's max_degree: report it
            if (atomicCAS(&p.ctl->status, CSG_OK, CSG_ERR_ARG) == CSG_OK) p.ctl->where = -1;
            d = min(d, kPRing - 1);
        }
        int* ring = lring + i * kPRing;
        ring[0] = v;
        for (int j = 0; j < d; ++j) ring[1 + j] = __ldg(p.nb + b + j);
        lnring[i] = d + 1;
        lvid[i] = v;
    }
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        const int lb = owned_below(__ldg(p.level_begin + l), c, nc), le = owned_below(__ldg(p.level_end + l), c, nc);
        lbeg[l] = lb;
        lend[l] = le;
        for (int i = lb; i < le; ++i) llev[i] = l;
    }
    for (int v = tid; v < p.n; v += nthreads) {
        const float4 q = ld4(p.work, v);
        csg::st_word(p.pub + 4LL * v, csg::make_word(q.x, 0u));
        csg::st_word(p.pub + 4LL * v + 1, csg::make_word(q.y, 0u));
        csg::st_word(p.pub + 4LL * v + 2, csg::make_word(q.z, 0u));
    }
    unsigned int phase = 0;
    int barrier_id = 0;
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    if (csg::ld_relaxed_gpu(&p.ctl->status) != CSG_OK) return;  // a ring overflow: same answer in every CTA
    const int span = (p.passes - 1) * D;  // host guarantees span + L < 2^31
    const int nsteps = span + L;
    int r = 0;
    for (int t = 0; t < nsteps; ++t, r = (r + 1 == D) ? 0 : r + 1) {
        int lo = t - span;
        if (lo < r) lo = r;
        const int hi = t < L ? t : (L - 1) - ((L - 1 - r) % D + D) % D;
        if (hi < lo) continue;
        const int i0 = lbeg[lo], i1 = lend[hi];
        int ib[kMaxSegments];
#pragma unroll
        for (int k = 1; k < kMaxSegments; ++k) {
            ib[k] = 0;
            if (k < p.n_segments) {
                const int m = t - p.seg[k].first_pass * D;
                ib[k] = m < lo ? i0 : (m >= hi ? i1 : lend[m]);
            }
        }
        for (int base = i0 + warp_first_group; base < i1; base += groups) {
            const int i = base + my_group;
            int v = -1, nring = 0, sg = 0;
            unsigned int pass = 0;
            const int* ring = nullptr;
            if (i < i1) {
                v = lvid[i];
                nring = lnring[i];
                ring = lring + i * kPRing;
                pass = static_cast<unsigned int>((t - llev[i]) / D);
#pragma unroll
                for (int k = 1; k < kMaxSegments; ++k) sg += i < ib[k];
            }
            if (!pass_vertex_df<G>(p, v, ring, nring, sg, pass, stage, pos)) return;
        }
    }
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    for (int v = tid; v < p.n; v += nthreads) {
        const unsigned long long* w = p.pub + 4LL * v;
        __stcg(p.work + v, make_float4(csg::word_value(csg::ld_word(w)), csg::word_value(csg::ld_word(w + 1)),
                                       csg::word_value(csg::ld_word(w + 2)), 0.0f));
    }
}

// ---------------------------------------------------------------- per-stage steps

__global__ void k_pack(const float* __restrict__ points, float4* __restrict__ work, int n) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) work[v] = make_float4(points[3 * v], points[3 * v + 1], points[3 * v + 2], 0.0f);
}

__global__ void k_unpack(const float4* __restrict__ work, float* __restrict__ points, int n) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const float4 q = work[v];
    points[3 * v] = q.x;
    points[3 * v + 1] = q.y;
    points[3 * v + 2] = q.z;
}

// ref = work; per run of kBlockSum vertices: coordinate sums, min, max.
__global__ void k_stage_partials(const float4* __restrict__ work, float4* __restrict__ ref, int n,
                                 double* __restrict__ partial) {
    const int run = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = run * kBlockSum;
    if (b >= n) return;
    double sum[3] = {0, 0, 0}, lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int v = b; v < n && v < b + kBlockSum; ++v) {
        const float4 q = work[v];
        ref[v] = q;
        const double x[3] = {q.x, q.y, q.z};
        for (int k = 0; k < 3; ++k) {
            sum[k] = __dadd_rn(sum[k], x[k]);
            lo[k] = fmin(lo[k], x[k]);
            hi[k] = fmax(hi[k], x[k]);
        }
    }
    double* out = partial + 9LL * run;
    for (int k = 0; k < 3; ++k) {
        out[k] = sum[k];
        out[3 + k] = lo[k];
        out[6 + k] = hi[k];
    }
}

__global__ void k_stage_stats(const double* __restrict__ partial, int runs, int n, Stats* __restrict__ st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int k = 0; k < 3; ++k) {
        double sum = 0.0, lo = INFINITY, hi = -INFINITY;
        for (int r = 0; r < runs; ++r) {
            sum = __dadd_rn(sum, partial[9LL * r + k]);
            lo = fmin(lo, partial[9LL * r + 3 + k]);
            hi = fmax(hi, partial[9LL * r + 6 + k]);
        }
        st->mean[k] = __ddiv_rn(sum, static_cast<double>(n));
        st->lo[k] = lo;
        st->hi[k] = hi;
        const double ext = __dsub_rn(hi, lo);
        st->extent[k] = ext < 1.0e-20 ? 1.0e-20 : ext;
    }
}

__global__ void k_center(float4* __restrict__ work, int n, const Stats* __restrict__ st) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const float4 q = work[v];
    work[v] = make_float4(__double2float_rn(__dsub_rn(q.x, st->mean[0])), __double2float_rn(__dsub_rn(q.y, st->mean[1])),
                          __double2float_rn(__dsub_rn(q.z, st->mean[2])), 0.0f);
}

__global__ void k_face_areas(const float4* __restrict__ pos, const int* __restrict__ faces, int nf,
                             double* __restrict__ area) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const float4 a = pos[faces[3 * f]], b = pos[faces[3 * f + 1]], c = pos[faces[3 * f + 2]];
    const double e0x = __dsub_rn(b.x, a.x), e0y = __dsub_rn(b.y, a.y), e0z = __dsub_rn(b.z, a.z);
    const double e1x = __dsub_rn(c.x, a.x), e1y = __dsub_rn(c.y, a.y), e1z = __dsub_rn(c.z, a.z);
    const double cx = __dsub_rn(__dmul_rn(e0y, e1z), __dmul_rn(e0z, e1y));
    const double cy = __dsub_rn(__dmul_rn(e0z, e1x), __dmul_rn(e0x, e1z));
    const double cz = __dsub_rn(__dmul_rn(e0x, e1y), __dmul_rn(e0y, e1x));
    double s = __dmul_rn(0.5, __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), __dmul_rn(cz, cz))));
    if (isnan(s)) s = 0.0;
    area[f] = s;
}

__global__ void k_run_sums(const double* __restrict__ x, int n, double* __restrict__ partial) {
    const int run = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = run * kBlockSum;
    if (b >= n) return;
    double s = 0.0;
    for (int i = b; i < n && i < b + kBlockSum; ++i) s = __dadd_rn(s, x[i]);
    partial[run] = s;
}

__global__ void k_finish_sum(const double* __restrict__ partial, int runs, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int r = 0; r < runs; ++r) s = __dadd_rn(s, partial[r]);
    *out = s;
}

// Vertex areas: a third of each incident face, in (corner, face) order
// (inc = face << 2 | corner, sorted by corner then face).
__global__ void k_vertex_areas(const double* __restrict__ area, const int* __restrict__ inc_off,
                               const int* __restrict__ inc, int n, double* __restrict__ va) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double s = 0.0;
    for (int k = inc_off[v]; k < inc_off[v + 1]; ++k) s = __dadd_rn(s, csg::div3_rn(area[inc[k] >> 2]));
    va[v] = s;
}

__device__ __forceinline__ double dist3(const float4& a, const float4& b) {
    const double x = __dsub_rn(b.x, a.x), y = __dsub_rn(b.y, a.y), z = __dsub_rn(b.z, a.z);
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

// Distortion measure per vertex (surf2sphere.py:573-629).
__global__ void k_distortion(const float4* __restrict__ work, const float4* __restrict__ ref,
                             const int* __restrict__ nb_off, const int* __restrict__ nb,
                             const double* __restrict__ va_cur, const double* __restrict__ va_ref, int n,
                             const Stats* __restrict__ st, double* __restrict__ comp) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const float4 pv = work[v], rv = ref[v];
    double max_linear = 0.0;
    for (int k = nb_off[v]; k < nb_off[v + 1]; ++k) {
        const int u = nb[k];
        const double rd = dist3(rv, ref[u]);
        const double ratio = rd > 0.0 ? __ddiv_rn(dist3(pv, work[u]), rd) : 0.0;
        if (ratio > max_linear) max_linear = ratio;
    }
    double area_ratio;
    if (va_cur[v] > 0.0) area_ratio = __ddiv_rn(va_ref[v], va_cur[v]);
    else area_ratio = va_ref[v] != 0.0 ? 10000.0 : 1.0;
    if (area_ratio < 1.0e-8) area_ratio = 1.0e-8;
    const double ref_surface = st->ref_surface > 1.0e-30 ? st->ref_surface : 1.0e-30;
    comp[v] = __dmul_rn(__dmul_rn(max_linear, area_ratio), __ddiv_rn(st->cur_surface, ref_surface));
}

__global__ void k_select(const double* __restrict__ comp, const int* __restrict__ nb_off, const int* __restrict__ nb,
                         int n, double threshold, unsigned char* __restrict__ selected) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double s = comp[v];
    for (int k = nb_off[v]; k < nb_off[v + 1]; ++k) s = __dadd_rn(s, comp[nb[k]]);
    selected[v] = __ddiv_rn(s, static_cast<double>(nb_off[v + 1] - nb_off[v] + 1)) > threshold;
}

// ---------------------------------------------------------------- ellipsoid to sphere

// convert_ellipsoid_to_sphere_with_surface_area (surf2sphere.py:919-937) on the
// device: float32 bounds, float32 half-axes (|lo| + |hi|) / 2 clamped to 1e-20,
// then per vertex in float64 x / a, |x / a|, radius x / |x / a| / a, float32
// store (a zero-length vertex becomes the origin).  Min and max are exact in
// any order, so one CTA reduces them; the result equals the host arithmetic.
__global__ void k_ellipsoid_bounds(const float* __restrict__ p, int n, float* __restrict__ axes) {
    __shared__ float lo[3][32], hi[3][32];
    float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int v = threadIdx.x; v < n; v += blockDim.x)
        for (int k = 0; k < 3; ++k) {
            const float x = p[3LL * v + k];
            l[k] = fminf(l[k], x);
            h[k] = fmaxf(h[k], x);
        }
    for (int k = 0; k < 3; ++k)
        for (int off = 16; off >= 1; off >>= 1) {
            l[k] = fminf(l[k], __shfl_xor_sync(kFull, l[k], off));
            h[k] = fmaxf(h[k], __shfl_xor_sync(kFull, h[k], off));
        }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int k = 0; k < 3; ++k) {
            lo[k][warp] = l[k];
            hi[k][warp] = h[k];
        }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int k = threadIdx.x;
        float a = INFINITY, b = -INFINITY;
        for (int w = 0; w < (blockDim.x + 31) / 32; ++w) {
            a = fminf(a, lo[k][w]);
            b = fmaxf(b, hi[k][w]);
        }
        const float half = __fmul_rn(__fadd_rn(fabsf(a), fabsf(b)), 0.5f);
        axes[k] = half < 1.0e-20f ? 1.0e-20f : half;
    }
}

__global__ void k_ellipsoid_scale(float* __restrict__ p, int n, const float* __restrict__ axes, double radius) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double x[3], s[3];
    for (int k = 0; k < 3; ++k) {
        x[k] = p[3LL * v + k];
        s[k] = __ddiv_rn(x[k], static_cast<double>(axes[k]));
    }
    const double norm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(s[0], s[0]), __dmul_rn(s[1], s[1])), __dmul_rn(s[2], s[2])));
    for (int k = 0; k < 3; ++k) {
        const double r = norm != 0.0 ? __ddiv_rn(__ddiv_rn(__dmul_rn(radius, x[k]), norm), static_cast<double>(axes[k]))
                                     : 0.0;
        p[3LL * v + k] = __double2float_rn(r);
    }
}

// ---------------------------------------------------------------- host side

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct Layout {
    size_t ctl, work, pub, ref, area, va_ref, va_cur, comp, sel, partial, stats, total;
};

Layout layout(int n, int nf) {
    Layout L{};
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t here = at;
        at += align256(bytes);
        return here;
    };
    const size_t runs = (static_cast<size_t>(n > nf ? n : nf) + kBlockSum - 1) / kBlockSum;
    L.ctl = take(sizeof(csg::Control));
    L.work = take(16ULL * n);
    L.pub = take(32ULL * n);
    L.ref = take(16ULL * n);
    L.area = take(8ULL * nf);
    L.va_ref = take(8ULL * n);
    L.va_cur = take(8ULL * n);
    L.comp = take(8ULL * n);
    L.sel = take(static_cast<size_t>(n));
    L.partial = take(8ULL * 9 * runs);
    L.stats = take(sizeof(Stats));
    L.total = at;
    return L;
}

constexpr size_t kMaxTopologySmem = 160 * 1024;

template <int G, bool SMEM>
int launch_variant(const PassParams& params, int n_ctas, int threads, size_t smem, cudaStream_t s) {
    auto kernel = smooth_passes_kernel<G, SMEM>;
    int device = 0, sms = 0, per_sm = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (SMEM) CSG_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1 || n_ctas > per_sm * sms)
        return csg::fail(CSG_ERR_LAUNCH, "preprocess passes: %d CTAs x %d threads (%zu B smem) cannot be co-resident",
                         n_ctas, threads, smem);
    PassParams p = params;
    void* args[] = {&p};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(n_ctas), dim3(threads), args,
                                               smem, s));
    csg::note_launch();
    return CSG_OK;
}

template <int G>
int launch_dataflow(const PassParams& params, int n_ctas, int threads, size_t smem, cudaStream_t s) {
    auto kernel = smooth_passes_df<G>;
    int device = 0, sms = 0, per_sm = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CSG_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1 || n_ctas > per_sm * sms)
        return csg::fail(CSG_ERR_LAUNCH, "preprocess passes: %d CTAs x %d threads (%zu B smem) cannot be co-resident",
                         n_ctas, threads, smem);
    PassParams p = params;
    void* args[] = {&p};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(n_ctas), dim3(threads), args,
                                               smem, s));
    csg::note_launch();
    return CSG_OK;
}

template <int G>
int launch_passes(PassParams params, int n_ctas, int threads, cudaStream_t s) {
    int device = 0, sms = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (n_ctas <= 0) n_ctas = sms;
    params.nloc_max = (params.n + n_ctas - 1) / n_ctas;
    if (params.max_degree > 0 && params.max_degree + 1 <= kPRing) {
        const size_t smem = sizeof(float3) * (threads / G) * kPRing +
                            sizeof(int) * (static_cast<size_t>(params.nloc_max) * (kPRing + 3) +
                                           2 * static_cast<size_t>(params.n_levels));
        if (smem <= kMaxTopologySmem) return launch_dataflow<G>(params, n_ctas, threads, smem, s);
    }
    const size_t smem = sizeof(int) * (static_cast<size_t>(params.nloc_max) * (params.max_degree + 2) +
                                       2 * static_cast<size_t>(params.n_levels));
    if (params.max_degree > 0 && smem <= kMaxTopologySmem) return launch_variant<G, true>(params, n_ctas, threads, smem, s);
    return launch_variant<G, false>(params, n_ctas, threads, 0, s);
}

// The passes queued since the last launch, launched as one wavefront.
struct PassQueue {
    PassParams p;
    int n_ctas, threads, lanes;
    cudaStream_t s;

    int add(int passes, int kind, double value) {
        if (passes <= 0) return CSG_OK;
        if (p.n_segments == kMaxSegments) {
            const int rc = launch();
            if (rc) return rc;
        }
        Segment& g = p.seg[p.n_segments++];
        g.first_pass = p.passes;
        g.kind = kind;
        g.value = value;
        p.passes += passes;
        return CSG_OK;
    }

    int launch() {
        if (p.passes <= 0) return CSG_OK;
        // every launch counts its barrier arrivals from zero; the status word is
        // kept, so a launch after a timed-out one leaves at its first barrier
        CSG_CUDA_CHECK(cudaMemsetAsync(&p.ctl->arrivals, 0, sizeof(p.ctl->arrivals), s));
        int rc;
        switch (lanes) {
            case 4: rc = launch_passes<4>(p, n_ctas, threads, s); break;
            case 16: rc = launch_passes<16>(p, n_ctas, threads, s); break;
            default: rc = launch_passes<8>(p, n_ctas, threads, s); break;
        }
        p.passes = 0;
        p.n_segments = 0;
        return rc;
    }
};

inline unsigned blocks(long long n, int threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

}  // namespace

extern "C" {

int csg_ellipsoid_to_sphere(float* points, int n, double radius, void* scratch, size_t scratch_bytes,
                            csg_stream_t stream) {
    if (!points || n < 1 || !scratch || scratch_bytes < 16 || !(radius >= 0.0))
        return csg::fail(CSG_ERR_ARG, "ellipsoid to sphere: bad arguments (16 bytes of scratch)");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    auto* axes = static_cast<float*>(scratch);
    (csg::note_launch(), k_ellipsoid_bounds<<<1, 1024, 0, s>>>(points, n, axes));
    (csg::note_launch(), k_ellipsoid_scale<<<blocks(n, kThreads), kThreads, 0, s>>>(points, n, axes, radius));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

size_t csg_preprocess_scratch_bytes(int n_vertices, int n_faces) {
    if (n_vertices < 4 || n_faces < 4) return 0;
    return layout(n_vertices, n_faces).total;
}

int csg_surf2sphere_preprocess(float* points, int n, const int32_t* faces, int nf, const int32_t* nb_off,
                               const int32_t* nb, const int32_t* inc_off, const int32_t* inc, const int32_t* order,
                               const int32_t* level_begin, const int32_t* level_end, int n_levels, int level_stride,
                               int max_degree, int stop_at, void* scratch, size_t scratch_bytes, int n_ctas,
                               int threads_per_cta, int lanes_per_vertex, double timeout_s, csg_stream_t stream) {
    if (!points || n < 4 || !faces || nf < 4 || !nb_off || !nb || !inc_off || !inc || !order || !level_begin ||
        !level_end || n_levels < 1 || level_stride < 1 || max_degree < 0 || stop_at < 1 || stop_at > 5 || !scratch)
        return csg::fail(CSG_ERR_ARG, "preprocess: bad arguments (stop_at 1..5)");
    if (threads_per_cta <= 0) threads_per_cta = 512;
    if (threads_per_cta % 32 || threads_per_cta > 512) return csg::fail(CSG_ERR_ARG, "preprocess: threads 32..512, x32");
    if (lanes_per_vertex <= 0) lanes_per_vertex = 8;
    if (lanes_per_vertex != 4 && lanes_per_vertex != 8 && lanes_per_vertex != 16)
        return csg::fail(CSG_ERR_ARG, "preprocess: lanes_per_vertex must be 4, 8 or 16");
    if (timeout_s <= 0.0) timeout_s = 2.0;
    const Layout L = layout(n, nf);
    if (scratch_bytes < L.total) return csg::fail(CSG_ERR_ARG, "preprocess: scratch too small");
    const double factor = nf > 350000 ? static_cast<double>(nf) / 350000.0 : 1.0;
    // every launch's span (passes - 1) * stride + levels must stay below 2^31
    // steps; a launch holds at most kMaxSegments segments of <= 60 factor passes
    if (kMaxSegments * std::nearbyint(factor * 60.0) * static_cast<double>(level_stride) + n_levels >= 2147483647.0)
        return csg::fail(CSG_ERR_ARG, "preprocess: schedule too long");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(scratch);
    auto* ctl = reinterpret_cast<csg::Control*>(base + L.ctl);
    auto* work = reinterpret_cast<float4*>(base + L.work);
    auto* ref = reinterpret_cast<float4*>(base + L.ref);
    auto* area = reinterpret_cast<double*>(base + L.area);
    auto* va_ref = reinterpret_cast<double*>(base + L.va_ref);
    auto* va_cur = reinterpret_cast<double*>(base + L.va_cur);
    auto* comp = reinterpret_cast<double*>(base + L.comp);
    auto* sel = reinterpret_cast<unsigned char*>(base + L.sel);
    auto* partial = reinterpret_cast<double*>(base + L.partial);
    auto* st = reinterpret_cast<Stats*>(base + L.stats);
    CSG_CUDA_CHECK(cudaMemsetAsync(ctl, 0, sizeof(csg::Control), s));
    (csg::note_launch(), k_pack<<<blocks(n, kThreads), kThreads, 0, s>>>(points, work, n));
    PassQueue q{};
    q.p.work = work;
    q.p.pub = reinterpret_cast<unsigned long long*>(base + L.pub);
    q.p.nb_off = nb_off;
    q.p.nb = nb;
    q.p.selected = sel;
    q.p.st = st;
    q.p.order = order;
    q.p.level_begin = level_begin;
    q.p.level_end = level_end;
    q.p.ctl = ctl;
    q.p.n = n;
    q.p.n_levels = n_levels;
    q.p.stride = level_stride;
    q.p.max_degree = max_degree;
    q.p.timeout_ns = static_cast<unsigned long long>(timeout_s * 1e9);
    q.n_ctas = n_ctas;
    q.threads = threads_per_cta;
    q.lanes = lanes_per_vertex;
    q.s = s;
    const int vruns = (n + kBlockSum - 1) / kBlockSum, fruns = (nf + kBlockSum - 1) / kBlockSum;
    // One launch runs at most: the previous cycle's selected passes, this
    // cycle's passes and the inflation.  Global steps (stage statistics, the
    // distortion selection) end a launch.
    for (int si = 0; si < stop_at; ++si) {
        const StageSpec spec = kStages[si];
        const int iterations = static_cast<int>(std::nearbyint(factor * spec.iterations));
        const int finger = static_cast<int>(std::nearbyint(factor * spec.finger_iterations));
        (csg::note_launch(), k_stage_partials<<<blocks(vruns, kThreads), kThreads, 0, s>>>(work, ref, n, partial));
        (csg::note_launch(), k_stage_stats<<<1, 32, 0, s>>>(partial, vruns, n, st));
        (csg::note_launch(), k_center<<<blocks(n, kThreads), kThreads, 0, s>>>(work, n, st));
        (csg::note_launch(), k_face_areas<<<blocks(nf, kThreads), kThreads, 0, s>>>(ref, faces, nf, area));
        (csg::note_launch(), k_run_sums<<<blocks(fruns, kThreads), kThreads, 0, s>>>(area, nf, partial));
        (csg::note_launch(), k_finish_sum<<<1, 32, 0, s>>>(partial, fruns, &st->ref_surface));
        (csg::note_launch(), k_vertex_areas<<<blocks(n, kThreads), kThreads, 0, s>>>(area, inc_off, inc, n, va_ref));
        const double delta = spec.inflation - 1.0;
        for (int cycle = 0; cycle < spec.cycles; ++cycle) {
            int rc = q.add(iterations - 1, kSmoothAll, spec.strength);
            if (!rc) rc = q.add(1, kInflate, delta);
            if (rc) return rc;
            if (finger > 0) {
                rc = q.launch();
                if (rc) return rc;
                (csg::note_launch(), k_face_areas<<<blocks(nf, kThreads), kThreads, 0, s>>>(work, faces, nf, area));
                (csg::note_launch(), k_run_sums<<<blocks(fruns, kThreads), kThreads, 0, s>>>(area, nf, partial));
                (csg::note_launch(), k_finish_sum<<<1, 32, 0, s>>>(partial, fruns, &st->cur_surface));
                (csg::note_launch(), k_vertex_areas<<<blocks(n, kThreads), kThreads, 0, s>>>(area, inc_off, inc, n,
                                                                                         va_cur));
                (csg::note_launch(), k_distortion<<<blocks(n, kThreads), kThreads, 0, s>>>(work, ref, nb_off, nb, va_cur,
                                                                                       va_ref, n, st, comp));
                (csg::note_launch(), k_select<<<blocks(n, kThreads), kThreads, 0, s>>>(comp, nb_off, nb, n,
                                                                                   spec.threshold, sel));
                rc = q.add(finger - 1, kSmoothSelected, spec.finger_strength);
                if (rc) return rc;
            }
        }
        int rc = q.launch();
        if (rc) return rc;
    }
    (csg::note_launch(), k_unpack<<<blocks(n, kThreads), kThreads, 0, s>>>(work, points, n));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

}  // extern "C"
