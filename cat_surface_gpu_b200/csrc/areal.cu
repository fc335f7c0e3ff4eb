// Surf2Sphere ordered area-smoothing sweeps as ONE persistent cooperative
// kernel for sm_100a.
//
// Semantics follow the reference's ordered Gauss-Seidel sweeps
// (src/cat_surface_gpu/surf2sphere.py:35-280 and 1039-1092): every vertex,
// in index order, moves to the area-weighted centroid of its incident faces
// (faces in ascending id, areas clamped to [0, 1]); after sweep s with
// s % project_every == 0 all points are projected to `radius`.
//
// Schedule: instead of one launch per dependency level per sweep (the
// reference launches sum(levels) x 4,999 kernels), vertex v of sweep s runs at
// wavefront step s * stride + level(v) inside one launch.  With
// stride = 1 + max_{edges v<w} (level(w) - level(v)) every read sees exactly
// the value the sequential order would see (lower neighbours: this sweep;
// higher neighbours: previous sweep), so the in-place buffer needs no copy.
// Steps are separated by a bounded grid barrier; projections drain the
// wavefront (one barrier before and after).
//
// Data layout: positions live in a float4 (or double4) working copy in HBM
// (L2-resident for cortical meshes), read with 16-byte ld.global.cg loads so
// no stale L1 line can be observed across steps.  Each vertex's incident
// faces are stored CSR-contiguous as int4 {v0, v1, v2, face}: a group of G
// lanes reads G consecutive slots (coalesced), computes one face per lane and
// accumulates the per-face terms in slot order through warp shuffles, which
// keeps the reference's sequential accumulation order exactly.
//
// Arithmetic: CSG_ARITH_CAT reproduces the reference's mixed precision
// (float32 edge/cross/sum-of-squares, float64 sqrt/centre/accumulate/divide,
// float32 store) with one IEEE rounding per operation (explicit _rn
// intrinsics, no contraction), so results are bit-identical to the CPU
// restatement compiled with -ffp-contract=off.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "common.cuh"
#include "errors.h"

namespace {

constexpr unsigned kFull = 0xffffffffu;

struct ArealParams {
    void* points;  // caller's [n,3] float32 or float64
    void* work;    // float4[n] or double4[n] working copy (scratch)
    csg::Control* ctl;
    const int4* slot_tri;
    const int* slot_off;
    const int* order;
    const int* level_begin;
    const int* level_end;
    int n;
    int n_levels;
    int stride;
    int max_degree;
    int nloc_max;  // vertices owned by one CTA (set at launch)
    int iterations;
    int project_every;
    int allow_dataflow;  // float32 modes: published (value, version) words instead of per-step barriers
    double radius;
    unsigned long long timeout_ns;
};

struct alignas(32) D4 {
    double x, y, z, w;
};

template <int MODE>
struct Traits;

// CAT mixed: float32 storage, float64 accumulation.
template <>
struct Traits<CSG_ARITH_CAT> {
    using Store = float4;
    using Acc = double;
    struct P3 {
        float x, y, z;
    };
    static __device__ __forceinline__ P3 load(const void* w, int v) {
        float4 q = __ldcg(static_cast<const float4*>(w) + v);
        return {q.x, q.y, q.z};
    }
    static __device__ __forceinline__ void face(const P3& a, const P3& b, const P3& c, double& area, double& mx,
                                                double& my, double& mz) {
        float e0x = __fsub_rn(b.x, a.x), e0y = __fsub_rn(b.y, a.y), e0z = __fsub_rn(b.z, a.z);
        float e1x = __fsub_rn(c.x, a.x), e1y = __fsub_rn(c.y, a.y), e1z = __fsub_rn(c.z, a.z);
        float cx = __fsub_rn(__fmul_rn(e0y, e1z), __fmul_rn(e0z, e1y));
        float cy = __fsub_rn(__fmul_rn(e0z, e1x), __fmul_rn(e0x, e1z));
        float cz = __fsub_rn(__fmul_rn(e0x, e1y), __fmul_rn(e0y, e1x));
        float sq = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
        area = __dmul_rn(0.5, __dsqrt_rn(static_cast<double>(sq)));
        mx = csg::div3_rn(__dadd_rn(__dadd_rn((double)a.x, (double)b.x), (double)c.x));
        my = csg::div3_rn(__dadd_rn(__dadd_rn((double)a.y, (double)b.y), (double)c.y));
        mz = csg::div3_rn(__dadd_rn(__dadd_rn((double)a.z, (double)b.z), (double)c.z));
        area = area > 0.0 ? area : 0.0;
        area = area < 1.0 ? area : 1.0;
    }
    static __device__ __forceinline__ void store(void* w, int v, double total, double wx, double wy, double wz) {
        double safe = total > 1.0e-20 ? total : 1.0e-20;
        float4 q = make_float4(__double2float_rn(__ddiv_rn(wx, safe)), __double2float_rn(__ddiv_rn(wy, safe)),
                               __double2float_rn(__ddiv_rn(wz, safe)), 0.0f);
        __stcg(static_cast<float4*>(w) + v, q);
    }
    static __device__ __forceinline__ P3 project_p3(const P3& q, double radius) {
        float sq = __fadd_rn(__fadd_rn(__fmul_rn(q.x, q.x), __fmul_rn(q.y, q.y)), __fmul_rn(q.z, q.z));
        double norm = __dsqrt_rn(static_cast<double>(sq));
        double scale = __ddiv_rn(radius, norm > 1.0e-20 ? norm : 1.0e-20);
        return {__double2float_rn(__dmul_rn((double)q.x, scale)), __double2float_rn(__dmul_rn((double)q.y, scale)),
                __double2float_rn(__dmul_rn((double)q.z, scale))};
    }
    static __device__ __forceinline__ void project(void* w, int v, double radius) {
        const P3 q = project_p3(load(w, v), radius);
        __stcg(static_cast<float4*>(w) + v, make_float4(q.x, q.y, q.z, 0.0f));
    }
    static __device__ __forceinline__ void pack(const void* in, void* w, int v) {
        const float* p = static_cast<const float*>(in) + 3LL * v;
        static_cast<float4*>(w)[v] = make_float4(p[0], p[1], p[2], 0.0f);
    }
    static __device__ __forceinline__ void unpack(const void* w, void* out, int v) {
        float4 q = __ldcg(static_cast<const float4*>(w) + v);
        float* p = static_cast<float*>(out) + 3LL * v;
        p[0] = q.x;
        p[1] = q.y;
        p[2] = q.z;
    }
};

// Plain float32 storage and arithmetic.
template <>
struct Traits<CSG_ARITH_FP32> {
    using Acc = float;
    using P3 = Traits<CSG_ARITH_CAT>::P3;
    static __device__ __forceinline__ P3 load(const void* w, int v) { return Traits<CSG_ARITH_CAT>::load(w, v); }
    static __device__ __forceinline__ void face(const P3& a, const P3& b, const P3& c, float& area, float& mx,
                                                float& my, float& mz) {
        float e0x = __fsub_rn(b.x, a.x), e0y = __fsub_rn(b.y, a.y), e0z = __fsub_rn(b.z, a.z);
        float e1x = __fsub_rn(c.x, a.x), e1y = __fsub_rn(c.y, a.y), e1z = __fsub_rn(c.z, a.z);
        float cx = __fsub_rn(__fmul_rn(e0y, e1z), __fmul_rn(e0z, e1y));
        float cy = __fsub_rn(__fmul_rn(e0z, e1x), __fmul_rn(e0x, e1z));
        float cz = __fsub_rn(__fmul_rn(e0x, e1y), __fmul_rn(e0y, e1x));
        float sq = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
        area = __fmul_rn(0.5f, __fsqrt_rn(sq));
        mx = __fdiv_rn(__fadd_rn(__fadd_rn(a.x, b.x), c.x), 3.0f);
        my = __fdiv_rn(__fadd_rn(__fadd_rn(a.y, b.y), c.y), 3.0f);
        mz = __fdiv_rn(__fadd_rn(__fadd_rn(a.z, b.z), c.z), 3.0f);
        area = area > 0.0f ? area : 0.0f;
        area = area < 1.0f ? area : 1.0f;
    }
    static __device__ __forceinline__ void store(void* w, int v, float total, float wx, float wy, float wz) {
        float safe = total > 1.0e-20f ? total : 1.0e-20f;
        __stcg(static_cast<float4*>(w) + v,
               make_float4(__fdiv_rn(wx, safe), __fdiv_rn(wy, safe), __fdiv_rn(wz, safe), 0.0f));
    }
    static __device__ __forceinline__ P3 project_p3(const P3& q, double radius) {
        const float r = static_cast<float>(radius);
        float sq = __fadd_rn(__fadd_rn(__fmul_rn(q.x, q.x), __fmul_rn(q.y, q.y)), __fmul_rn(q.z, q.z));
        float norm = __fsqrt_rn(sq);
        float scale = __fdiv_rn(r, norm > 1.0e-20f ? norm : 1.0e-20f);
        return {__fmul_rn(q.x, scale), __fmul_rn(q.y, scale), __fmul_rn(q.z, scale)};
    }
    static __device__ __forceinline__ void project(void* w, int v, double radius) {
        const P3 q = project_p3(load(w, v), radius);
        __stcg(static_cast<float4*>(w) + v, make_float4(q.x, q.y, q.z, 0.0f));
    }
    static __device__ __forceinline__ void pack(const void* in, void* w, int v) { Traits<CSG_ARITH_CAT>::pack(in, w, v); }
    static __device__ __forceinline__ void unpack(const void* w, void* out, int v) {
        Traits<CSG_ARITH_CAT>::unpack(w, out, v);
    }
};

// Float64 storage and arithmetic.
template <>
struct Traits<CSG_ARITH_FP64> {
    using Acc = double;
    struct P3 {
        double x, y, z;
    };
    static __device__ __forceinline__ P3 load(const void* w, int v) {
        const double2* base = reinterpret_cast<const double2*>(static_cast<const D4*>(w) + v);
        double2 xy = __ldcg(base);
        double2 zw = __ldcg(base + 1);
        return {xy.x, xy.y, zw.x};
    }
    static __device__ __forceinline__ void face(const P3& a, const P3& b, const P3& c, double& area, double& mx,
                                                double& my, double& mz) {
        double e0x = __dsub_rn(b.x, a.x), e0y = __dsub_rn(b.y, a.y), e0z = __dsub_rn(b.z, a.z);
        double e1x = __dsub_rn(c.x, a.x), e1y = __dsub_rn(c.y, a.y), e1z = __dsub_rn(c.z, a.z);
        double cx = __dsub_rn(__dmul_rn(e0y, e1z), __dmul_rn(e0z, e1y));
        double cy = __dsub_rn(__dmul_rn(e0z, e1x), __dmul_rn(e0x, e1z));
        double cz = __dsub_rn(__dmul_rn(e0x, e1y), __dmul_rn(e0y, e1x));
        double sq = __dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), __dmul_rn(cz, cz));
        area = __dmul_rn(0.5, __dsqrt_rn(sq));
        mx = csg::div3_rn(__dadd_rn(__dadd_rn(a.x, b.x), c.x));
        my = csg::div3_rn(__dadd_rn(__dadd_rn(a.y, b.y), c.y));
        mz = csg::div3_rn(__dadd_rn(__dadd_rn(a.z, b.z), c.z));
        area = area > 0.0 ? area : 0.0;
        area = area < 1.0 ? area : 1.0;
    }
    static __device__ __forceinline__ void write(void* w, int v, double x, double y, double z) {
        double2* base = reinterpret_cast<double2*>(static_cast<D4*>(w) + v);
        __stcg(base, make_double2(x, y));
        __stcg(base + 1, make_double2(z, 0.0));
    }
    static __device__ __forceinline__ void store(void* w, int v, double total, double wx, double wy, double wz) {
        double safe = total > 1.0e-20 ? total : 1.0e-20;
        write(w, v, __ddiv_rn(wx, safe), __ddiv_rn(wy, safe), __ddiv_rn(wz, safe));
    }
    static __device__ __forceinline__ void project(void* w, int v, double radius) {
        P3 q = load(w, v);
        double sq = __dadd_rn(__dadd_rn(__dmul_rn(q.x, q.x), __dmul_rn(q.y, q.y)), __dmul_rn(q.z, q.z));
        double norm = __dsqrt_rn(sq);
        double scale = __ddiv_rn(radius, norm > 1.0e-20 ? norm : 1.0e-20);
        write(w, v, __dmul_rn(q.x, scale), __dmul_rn(q.y, scale), __dmul_rn(q.z, scale));
    }
    static __device__ __forceinline__ void pack(const void* in, void* w, int v) {
        const double* p = static_cast<const double*>(in) + 3LL * v;
        write(w, v, p[0], p[1], p[2]);
    }
    static __device__ __forceinline__ void unpack(const void* w, void* out, int v) {
        P3 q = load(w, v);
        double* p = static_cast<double*>(out) + 3LL * v;
        p[0] = q.x;
        p[1] = q.y;
        p[2] = q.z;
    }
};

template <typename T>
__device__ __forceinline__ T dadd(T a, T b);
template <>
__device__ __forceinline__ double dadd<double>(double a, double b) { return __dadd_rn(a, b); }
template <>
__device__ __forceinline__ float dadd<float>(float a, float b) { return __fadd_rn(a, b); }
template <typename T>
__device__ __forceinline__ T dmul(T a, T b);
template <>
__device__ __forceinline__ double dmul<double>(double a, double b) { return __dmul_rn(a, b); }
template <>
__device__ __forceinline__ float dmul<float>(float a, float b) { return __fmul_rn(a, b); }

// One vertex update by a group of G lanes.  All 32 lanes of the warp must
// call this together (warp shuffles); inactive groups pass v < 0.  `tri`
// points at the vertex's incident-face slots (shared or global memory).
//
// float64 accumulation (CAT and FP64 modes): every lane computes one face's
// area and area-weighted centre products and stages them in shared memory;
// lanes 0, 1 and 2 of the group then each sum, in slot order, the area
// total and one coordinate's weighted sum and divide it -- three dependent
// chains and three divides in parallel instead of one lane doing all four
// sums and three divides.  The arithmetic is unchanged: same products, same
// order of additions.
template <int MODE, int G, bool SMEM>
__device__ __forceinline__ void update_vertex(const ArealParams& p, int v, const int4* tri, int deg,
                                              double (*stage)[32]) {
    using T = Traits<MODE>;
    using Acc = typename T::Acc;
    const int lane = threadIdx.x & 31;
    const int glane = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    if (v < 0) deg = 0;
    const int wdeg = __reduce_max_sync(kFull, deg);
    if constexpr (sizeof(Acc) == 8) {
        double total = 0, wsum = 0;
        const double* mine = stage[1 + (glane < 3 ? glane : 0)];
        for (int c0 = 0; c0 < wdeg; c0 += G) {
            const int j = c0 + glane;
            double fa = 0, fx = 0, fy = 0, fz = 0;
            if (j < deg) {
                const int4 t = SMEM ? tri[j] : __ldg(tri + j);
                auto a = T::load(p.work, t.x);
                auto b = T::load(p.work, t.y);
                auto c = T::load(p.work, t.z);
                double mx, my, mz;
                T::face(a, b, c, fa, mx, my, mz);
                fx = __dmul_rn(fa, mx);
                fy = __dmul_rn(fa, my);
                fz = __dmul_rn(fa, mz);
            }
            stage[0][lane] = fa;
            stage[1][lane] = fx;
            stage[2][lane] = fy;
            stage[3][lane] = fz;
            __syncwarp();
            if (glane < 3) {
                const int n = min(G, deg - c0);
#pragma unroll
                for (int q = 0; q < G; ++q) {
                    if (q < n) {  // slot order == ascending face id
                        total = __dadd_rn(total, stage[0][gbase + q]);
                        wsum = __dadd_rn(wsum, mine[gbase + q]);
                    }
                }
            }
            __syncwarp();
        }
        const bool write = v >= 0 && total > 0.0;
        const double safe = total > 1.0e-20 ? total : 1.0e-20;
        const double comp = (glane < 3 && write) ? __ddiv_rn(wsum, safe) : 0.0;
        if constexpr (MODE == CSG_ARITH_CAT) {
            const float cf = __double2float_rn(comp);
            const float cy = __shfl_sync(kFull, cf, gbase + 1);
            const float cz = __shfl_sync(kFull, cf, gbase + 2);
            if (write && glane == 0) __stcg(static_cast<float4*>(p.work) + v, make_float4(cf, cy, cz, 0.0f));
        } else {
            const double cy = __shfl_sync(kFull, comp, gbase + 1);
            const double cz = __shfl_sync(kFull, comp, gbase + 2);
            if (write && glane == 0) T::write(p.work, v, comp, cy, cz);
        }
    } else {
        Acc total = 0, wx = 0, wy = 0, wz = 0;
        for (int c0 = 0; c0 < wdeg; c0 += G) {
            const int j = c0 + glane;
            Acc fa = 0, fx = 0, fy = 0, fz = 0;
            if (j < deg) {
                const int4 t = SMEM ? tri[j] : __ldg(tri + j);
                auto a = T::load(p.work, t.x);
                auto b = T::load(p.work, t.y);
                auto c = T::load(p.work, t.z);
                T::face(a, b, c, fa, fx, fy, fz);
            }
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const Acc a = __shfl_sync(kFull, fa, gbase + q);
                const Acc x = __shfl_sync(kFull, fx, gbase + q);
                const Acc y = __shfl_sync(kFull, fy, gbase + q);
                const Acc z = __shfl_sync(kFull, fz, gbase + q);
                if (c0 + q < deg) {  // slot order == ascending face id
                    total = dadd<Acc>(total, a);
                    wx = dadd<Acc>(wx, dmul<Acc>(a, x));
                    wy = dadd<Acc>(wy, dmul<Acc>(a, y));
                    wz = dadd<Acc>(wz, dmul<Acc>(a, z));
                }
            }
        }
        if (v >= 0 && glane == 0 && total > Acc(0)) T::store(p.work, v, total, wx, wy, wz);
    }
}

// Number of positions c, c + nc, c + 2 nc, ... that lie below `bound`.
__device__ __forceinline__ int owned_below(int bound, int c, int nc) { return bound > c ? (bound - c + nc - 1) / nc : 0; }

// Vertex ownership: CTA c owns the vertices at positions c, c + n_ctas, ...
// of `order`, so every dependency level (a contiguous run of `order`) is
// spread evenly over all CTAs and a CTA always updates the same vertices.
// With SMEM the CTA copies those vertices' incident-face slots into shared
// memory once; each wavefront step then only gathers positions from L2.
template <int MODE, int G, bool SMEM>
__global__ void __launch_bounds__(512) areal_sweeps_kernel(ArealParams p) {
    using T = Traits<MODE>;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double stage_all[512 / 32][4][32];  // per-warp staging of face terms (float64 modes)
    double (*stage)[32] = stage_all[threadIdx.x >> 5];
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthreads = gridDim.x * blockDim.x;
    const int c = blockIdx.x;
    const int nc = gridDim.x;
    const int groups = blockDim.x / G;
    const int warp_first_group = (threadIdx.x >> 5) * (32 / G);
    const int my_group = (threadIdx.x & 31) / G;
    const int nloc = owned_below(p.n, c, nc);
    const int L = p.n_levels;
    const int D = p.stride;
    // shared-memory image (SMEM only): face slots, vertex ids and degrees of
    // the owned vertices, then per-level owned ranges and per-residue top level
    int4* ltri = reinterpret_cast<int4*>(smem);
    int* lvid = reinterpret_cast<int*>(ltri + (SMEM ? p.nloc_max * p.max_degree : 0));
    int* ldeg = lvid + p.nloc_max;
    int* lbeg = ldeg + p.nloc_max;
    int* lend = lbeg + L;
    int* hitop = lend + L;
    unsigned int phase = 0;
    int barrier_id = 0;

    if (SMEM) {
        for (int i = threadIdx.x; i < nloc; i += blockDim.x) {
            const int v = __ldg(p.order + c + i * nc);
            const int s0 = __ldg(p.slot_off + v);
            int d = __ldg(p.slot_off + v + 1) - s0;
            if (d < 0 || d > p.max_degree) {  // plan and max_degree disagree: report, stay inside the image
                if (atomicCAS(&p.ctl->status, CSG_OK, CSG_ERR_ARG) == CSG_OK) p.ctl->where = -3;
                d = 0;
            }
            lvid[i] = v;
            ldeg[i] = d;
            for (int j = 0; j < d; ++j) ltri[i * p.max_degree + j] = __ldg(p.slot_tri + s0 + j);
        }
        for (int l = threadIdx.x; l < L; l += blockDim.x) {
            lbeg[l] = owned_below(__ldg(p.level_begin + l), c, nc);
            lend[l] = owned_below(__ldg(p.level_end + l), c, nc);
        }
        for (int r = threadIdx.x; r < D; r += blockDim.x) hitop[r] = (L - 1) - ((L - 1 - r) % D + D) % D;
    }
    for (int v = tid; v < p.n; v += nthreads) T::pack(p.points, p.work, v);
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    if (SMEM && csg::ld_relaxed_gpu(&p.ctl->status) != CSG_OK) return;  // a degree over max_degree: every CTA sees it

    const int last = p.iterations - 1;
    for (int start = 1; start <= last;) {
        int end = last;
        if (p.project_every > 0) end = min(last, ((start - 1) / p.project_every + 1) * p.project_every);
        const int S = end - start + 1;
        const int span = (S - 1) * D;        // host guarantees span + L < 2^31
        const int nsteps = span + L;
        int r = 0;                           // r == t mod D, kept incrementally
        for (int t = 0; t < nsteps; ++t, r = (r + 1 == D) ? 0 : r + 1) {
            // active levels: lo, lo + D, ..., hi (all congruent to t mod D)
            int hi, lo = t - span;
            if (lo < r) lo = r;
            int i0, i1;
            if (SMEM) {
                hi = t < L ? t : hitop[r];
                if (hi < lo) continue;  // no vertex of any sweep sits on this step
                i0 = lbeg[lo];
                i1 = lend[hi];
            } else {
                hi = t < L ? t : (L - 1) - ((L - 1 - r) % D + D) % D;
                if (hi < lo) continue;
                i0 = owned_below(__ldg(p.level_begin + lo), c, nc);
                i1 = owned_below(__ldg(p.level_end + hi), c, nc);
            }
            for (int base = i0 + warp_first_group; base < i1; base += groups) {
                const int i = base + my_group;
                int v = -1, deg = 0;
                const int4* tri = nullptr;
                if (i < i1) {
                    if (SMEM) {
                        v = lvid[i];
                        deg = ldeg[i];
                        tri = ltri + i * p.max_degree;
                    } else {
                        v = __ldg(p.order + c + i * nc);
                        const int s0 = __ldg(p.slot_off + v);
                        deg = __ldg(p.slot_off + v + 1) - s0;
                        tri = p.slot_tri + s0;
                    }
                }
                update_vertex<MODE, G, SMEM>(p, v, tri, deg, stage);
            }
            if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
        }
        if (p.project_every > 0 && end % p.project_every == 0) {
            for (int v = tid; v < p.n; v += nthreads) T::project(p.work, v, p.radius);
            if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
        }
        start = end + 1;
    }
    for (int v = tid; v < p.n; v += nthreads) T::unpack(p.work, p.points, v);
}

// ---------------------------------------------------------------------------
// Dataflow form of the sweeps (float32 storage modes).
//
// The grid barrier between wavefront steps is replaced by per-vertex versions.
// Each coordinate of each vertex is published as one 8-byte word
// (float32 bits | version << 32), version = the number of sweeps the vertex
// has completed; 8-byte aligned accesses are single-copy atomic, so a word
// read with a relaxed load carries a value and the version it belongs to.
// Sweep s of vertex v needs lower-index neighbours at version s and
// higher-index neighbours and v itself at version s - 1, and neither can be
// further ahead: a lower neighbour u cannot finish sweep s + 1 before v
// finishes sweep s (v > u is its higher neighbour), a higher neighbour w cannot
// finish sweep s before v does.  So once every word shows its required version
// the values are exactly the sequential Gauss-Seidel inputs, and the group
// polls its faces' words until they do.  Each group walks the same wavefront
// order as the barrier form (step t, then its share of the step's vertices),
// which keeps progress guaranteed: the earliest unfinished update's inputs are
// all finished.  The projections ride in the wavefront too (a second array
// of projected words, written as each epoch's last sweep is published), so
// one wavefront runs every sweep and grid barriers remain only at the start
// and the end.
// Every wait is bounded: on timeout (or another CTA's failure) the kernel
// records the status and leaves.

using csg::ld_word;
using csg::make_word;
using csg::st_word;
using csg::word_value;
using csg::word_version;

// words of vertex v: pub[4 v + k], k = 0, 1, 2 (coordinate k), 3 unused
template <typename P3>
__device__ __forceinline__ bool load_versioned(const unsigned long long* pub, int u, unsigned int need, P3& q) {
    const unsigned long long* w = pub + 4LL * u;
    const unsigned long long a = ld_word(w), b = ld_word(w + 1), c = ld_word(w + 2);
    q = {word_value(a), word_value(b), word_value(c)};
    return word_version(a) == need && word_version(b) == need && word_version(c) == need;
}

__device__ __forceinline__ bool wait_expired(const ArealParams& p, unsigned int& polls, unsigned long long& start) {
    return csg::warp_wait_expired(p.ctl, p.timeout_ns, polls, start);
}

// Ring of a vertex: itself, then the other vertices of its faces (at most
// kRingMax); each face slot is coded as three ring indices (8 bits each).
constexpr int kRingMax = 20;

// One vertex update of sweep s by a group of G lanes (all 32 lanes call it;
// inactive groups pass v < 0).  The group first polls the words of the ring --
// lane j loads members j, j + G, ... all at once, one round trip per poll --
// and stages the positions in shared memory (`pos`, kRingMax entries per
// group), then computes the faces exactly as update_vertex does (same
// arithmetic, slot order).  Lanes 0, 1, 2 publish coordinates 0, 1, 2.
// Returns false to abort.
template <int MODE, int G>
__device__ __forceinline__ bool update_vertex_df(const ArealParams& p, unsigned long long* pub,
                                                 const unsigned long long* prev, unsigned long long* proj_out, int v,
                                                 const int* ring, int nring, const int* code, int deg, unsigned int s,
                                                 double (*stage)[32], float3* pos) {
    using T = Traits<MODE>;
    using Acc = typename T::Acc;
    using P3 = typename T::P3;
    constexpr int kQ = (kRingMax + G - 1) / G;
    const int lane = threadIdx.x & 31;
    const int glane = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    if (v < 0) {
        deg = 0;
        nring = 0;
    }
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
                for (int k = 0; k < 3; ++k) w[q][k] = ld_word((who[q] < v ? pub : prev) + 4LL * who[q] + k);
        bool ok = true;
#pragma unroll
        for (int q = 0; q < kQ; ++q)
            if (who[q] >= 0) {
                const unsigned int need = who[q] < v ? s : s - 1;  // the vertex itself: s - 1
                ok = ok && word_version(w[q][0]) == need && word_version(w[q][1]) == need &&
                     word_version(w[q][2]) == need;
                pos[glane + q * G] = make_float3(word_value(w[q][0]), word_value(w[q][1]), word_value(w[q][2]));
            }
        if (__all_sync(kFull, ok)) break;
        if (wait_expired(p, polls, start)) return false;
    }
    __syncwarp();
    const int wdeg = __reduce_max_sync(kFull, deg);
    Acc total = 0, wx = 0, wy = 0, wz = 0;  // float path: every lane sums its group's faces
    double wsum = 0;                        // float64 path: lanes 0..2 sum one coordinate each
    for (int c0 = 0; c0 < wdeg; c0 += G) {
        const int j = c0 + glane;
        const bool face = j < deg;
        P3 a{}, b{}, c{};
        if (face) {
            const int cd = code[j];
            const float3 pa = pos[cd & 255], pb = pos[(cd >> 8) & 255], pc = pos[(cd >> 16) & 255];
            a = {pa.x, pa.y, pa.z};
            b = {pb.x, pb.y, pb.z};
            c = {pc.x, pc.y, pc.z};
        }
        if constexpr (sizeof(Acc) == 8) {
            double fa = 0, fx = 0, fy = 0, fz = 0;
            if (face) {
                double mx, my, mz;
                T::face(a, b, c, fa, mx, my, mz);
                fx = __dmul_rn(fa, mx);
                fy = __dmul_rn(fa, my);
                fz = __dmul_rn(fa, mz);
            }
            stage[0][lane] = fa;
            stage[1][lane] = fx;
            stage[2][lane] = fy;
            stage[3][lane] = fz;
            __syncwarp();
            if (glane < 3) {
                const double* mine = stage[1 + glane];
                const int n = min(G, deg - c0);
#pragma unroll
                for (int q = 0; q < G; ++q) {
                    if (q < n) {  // slot order == ascending face id
                        total = __dadd_rn(total, stage[0][gbase + q]);
                        wsum = __dadd_rn(wsum, mine[gbase + q]);
                    }
                }
            }
            __syncwarp();
        } else {
            Acc fa = 0, fx = 0, fy = 0, fz = 0;
            if (face) T::face(a, b, c, fa, fx, fy, fz);
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const Acc aa = __shfl_sync(kFull, fa, gbase + q);
                const Acc x = __shfl_sync(kFull, fx, gbase + q);
                const Acc y = __shfl_sync(kFull, fy, gbase + q);
                const Acc z = __shfl_sync(kFull, fz, gbase + q);
                if (c0 + q < deg) {  // slot order == ascending face id
                    total = dadd<Acc>(total, aa);
                    wx = dadd<Acc>(wx, dmul<Acc>(aa, x));
                    wy = dadd<Acc>(wy, dmul<Acc>(aa, y));
                    wz = dadd<Acc>(wz, dmul<Acc>(aa, z));
                }
            }
        }
    }
    // a vertex that does not move republishes its own position (ring member 0)
    float value = 0.0f;
    if (v >= 0 && glane < 3) value = glane == 0 ? pos[0].x : (glane == 1 ? pos[0].y : pos[0].z);
    if constexpr (sizeof(Acc) == 8) {
        // total is summed by each of lanes 0..2 (same order, same value)
        if (v >= 0 && glane < 3 && total > 0.0) {
            const double safe = total > 1.0e-20 ? total : 1.0e-20;
            value = __double2float_rn(__ddiv_rn(wsum, safe));
        }
    } else {
        float nx = 0.0f, ny = 0.0f, nz = 0.0f;
        const bool moved = v >= 0 && glane == 0 && total > Acc(0);
        if (moved) {
            const float safe = total > 1.0e-20f ? total : 1.0e-20f;
            nx = __fdiv_rn(wx, safe);
            ny = __fdiv_rn(wy, safe);
            nz = __fdiv_rn(wz, safe);
        }
        const int m = __shfl_sync(kFull, moved ? 1 : 0, gbase);
        const float ny1 = __shfl_sync(kFull, ny, gbase);
        const float nz2 = __shfl_sync(kFull, nz, gbase);
        if (m) value = glane == 0 ? nx : (glane == 1 ? ny1 : nz2);
    }
    __syncwarp();  // every lane is done with `pos` before the next update overwrites it
    if (v >= 0 && glane < 3) st_word(pub + 4LL * v + glane, make_word(value, s));
    if (__any_sync(kFull, proj_out != nullptr && v >= 0)) {
        // sweep s ends a projection epoch: publish the projected point too (T::project_p3 of
        // the float32 values just published, as the separate projection pass computed it)
        const float px = __shfl_sync(kFull, value, gbase), py = __shfl_sync(kFull, value, gbase + 1),
                    pz = __shfl_sync(kFull, value, gbase + 2);
        if (proj_out != nullptr && v >= 0 && glane < 3) {
            const P3 q = T::project_p3(P3{px, py, pz}, p.radius);
            st_word(proj_out + 4LL * v + glane, make_word(glane == 0 ? q.x : (glane == 1 ? q.y : q.z), s));
        }
    }
    return true;
}

template <int MODE, int G>
__global__ void __launch_bounds__(512) areal_dataflow_kernel(ArealParams p) {
    using T = Traits<MODE>;
    using P3 = typename T::P3;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double stage_all[512 / 32][4][32];
    double (*stage)[32] = stage_all[threadIdx.x >> 5];
    unsigned long long* pub = static_cast<unsigned long long*>(p.work);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthreads = gridDim.x * blockDim.x;
    const int c = blockIdx.x;
    const int nc = gridDim.x;
    const int groups = blockDim.x / G;
    const int warp_first_group = (threadIdx.x >> 5) * (32 / G);
    const int my_group = (threadIdx.x & 31) / G;
    const int nloc = owned_below(p.n, c, nc);
    const int L = p.n_levels;
    const int D = p.stride;
    // shared-memory image: per warp, kRingMax staged positions per group; per
    // owned vertex its ring, ring size, face codes, id, degree and level; per
    // level the owned range; per residue the top level
    float3* wpos = reinterpret_cast<float3*>(smem) + (threadIdx.x >> 5) * (32 / G) * kRingMax;
    float3* pos = wpos + my_group * kRingMax;
    int* lring = reinterpret_cast<int*>(reinterpret_cast<float3*>(smem) + (blockDim.x / 32) * (32 / G) * kRingMax);
    int* lcode = lring + p.nloc_max * kRingMax;
    int* lnring = lcode + p.nloc_max * p.max_degree;
    int* lvid = lnring + p.nloc_max;
    int* ldeg = lvid + p.nloc_max;
    int* llev = ldeg + p.nloc_max;
    int* lbeg = llev + p.nloc_max;
    int* lend = lbeg + L;
    int* hitop = lend + L;
    unsigned int phase = 0;
    int barrier_id = 0;
    for (int i = threadIdx.x; i < nloc; i += blockDim.x) {
        const int v = __ldg(p.order + c + i * nc);
        const int s0 = __ldg(p.slot_off + v);
        int d = __ldg(p.slot_off + v + 1) - s0;
        if (d < 0 || d > p.max_degree) {  // plan and max_degree disagree: report, stay inside the image
            if (atomicCAS(&p.ctl->status, CSG_OK, CSG_ERR_ARG) == CSG_OK) p.ctl->where = -3;
            d = 0;
        }
        int* ring = lring + i * kRingMax;
        int nr = 1;
        ring[0] = v;
        for (int j = 0; j < d; ++j) {
            const int4 t = __ldg(p.slot_tri + s0 + j);
            const int u[3] = {t.x, t.y, t.z};
            int cd = 0;
            for (int k = 0; k < 3; ++k) {
                int at = 0;
                while (at < nr && ring[at] != u[k]) ++at;
                if (at == nr) {
                    if (nr == kRingMax) {  // the host sized kRingMax from max_degree; report, stay inside
                        if (atomicCAS(&p.ctl->status, CSG_OK, CSG_ERR_ARG) == CSG_OK) p.ctl->where = -1;
                        at = 0;
                    } else {
                        ring[nr++] = u[k];
                    }
                }
                cd |= at << (8 * k);
            }
            lcode[i * p.max_degree + j] = cd;
        }
        lnring[i] = nr;
        lvid[i] = v;
        ldeg[i] = d;
    }
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        const int b = owned_below(__ldg(p.level_begin + l), c, nc), e = owned_below(__ldg(p.level_end + l), c, nc);
        lbeg[l] = b;
        lend[l] = e;
        for (int i = b; i < e; ++i) llev[i] = l;
    }
    for (int r = threadIdx.x; r < D; r += blockDim.x) hitop[r] = (L - 1) - ((L - 1 - r) % D + D) % D;
    for (int v = tid; v < p.n; v += nthreads) {
        const float* q = static_cast<const float*>(p.points) + 3LL * v;
        for (int k = 0; k < 3; ++k) st_word(pub + 4LL * v + k, make_word(q[k], 0u));
        // projected words start at version 0, below any epoch's end: a word left
        // from an earlier call on the same scratch never satisfies a poll
        for (int k = 0; k < 3; ++k) st_word(pub + 4LL * p.n + 4LL * v + k, make_word(0.0f, 0u));
    }
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    // a ring overflow or a degree over max_degree: the same answer in every CTA
    if (csg::ld_relaxed_gpu(&p.ctl->status) != CSG_OK) return;

    // One wavefront over every sweep.  The projection after sweep b (b a multiple of
    // project_every) is applied by each vertex's group as it publishes sweep b, into
    // the second word array `proj`; the updates of sweep b + 1 read their
    // previous-sweep members (higher neighbours and the vertex itself) from there,
    // the updates of sweep b read the unprojected words.  The wavefront therefore
    // never drains at a projection.
    const int last = p.iterations - 1;
    unsigned long long* proj = pub + 4LL * p.n;
    if (last >= 1) {
        const int span = (last - 1) * D;  // host guarantees span + L < 2^31
        const int nsteps = span + L;
        int r = 0;
        for (int t = 0; t < nsteps; ++t, r = (r + 1 == D) ? 0 : r + 1) {
            int lo = t - span;
            if (lo < r) lo = r;
            const int hi = t < L ? t : hitop[r];
            if (hi < lo) continue;
            const int i0 = lbeg[lo], i1 = lend[hi];
            for (int base = i0 + warp_first_group; base < i1; base += groups) {
                const int i = base + my_group;
                int v = -1, deg = 0, nring = 0;
                unsigned int sweep = 0;
                const int* ring = nullptr;
                const int* code = nullptr;
                if (i < i1) {
                    v = lvid[i];
                    deg = ldeg[i];
                    nring = lnring[i];
                    ring = lring + i * kRingMax;
                    code = lcode + i * p.max_degree;
                    sweep = static_cast<unsigned int>(1 + (t - llev[i]) / D);
                }
                const bool after = p.project_every > 0 && sweep > 1 && (sweep - 1) % p.project_every == 0;
                const bool at = p.project_every > 0 && sweep > 0 && sweep % p.project_every == 0;
                if (!update_vertex_df<MODE, G>(p, pub, after ? proj : pub, at ? proj : nullptr, v, ring, nring, code,
                                               deg, sweep, stage, pos))
                    return;
            }
        }
    }
    if (csg::grid_barrier(p.ctl, phase, p.timeout_ns, barrier_id++)) return;
    const unsigned long long* result =
        (p.project_every > 0 && last >= 1 && last % p.project_every == 0) ? proj : pub;
    for (int v = tid; v < p.n; v += nthreads) {
        float* q = static_cast<float*>(p.points) + 3LL * v;
        for (int k = 0; k < 3; ++k) q[k] = word_value(ld_word(result + 4LL * v + k));
    }
}

constexpr size_t kMaxTopologySmem = 200 * 1024;

template <int MODE, int G, bool SMEM>
int launch_variant(ArealParams params, int n_ctas, int threads, size_t smem, cudaStream_t stream) {
    auto kernel = areal_sweeps_kernel<MODE, G, SMEM>;
    int device = 0, sms = 0, per_sm = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (SMEM) CSG_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1 || n_ctas > per_sm * sms)
        return csg::fail(CSG_ERR_LAUNCH, "areal sweeps: %d CTAs x %d threads (%zu B smem) cannot be co-resident (%d per SM, %d SMs)",
                         n_ctas, threads, smem, per_sm, sms);
    void* args[] = {&params};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(n_ctas), dim3(threads), args,
                                               smem, stream));
    csg::note_launch();
    return CSG_OK;
}

template <int MODE, int G>
int launch_dataflow(ArealParams params, int n_ctas, int threads, size_t smem, cudaStream_t stream) {
    auto kernel = areal_dataflow_kernel<MODE, G>;
    int device = 0, sms = 0, per_sm = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CSG_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1 || n_ctas > per_sm * sms)
        return csg::fail(CSG_ERR_LAUNCH, "areal sweeps: %d CTAs x %d threads (%zu B smem) cannot be co-resident (%d per SM, %d SMs)",
                         n_ctas, threads, smem, per_sm, sms);
    void* args[] = {&params};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(n_ctas), dim3(threads), args,
                                               smem, stream));
    csg::note_launch();
    return CSG_OK;
}

template <int MODE, int G>
int launch(ArealParams params, int n_ctas, int threads, cudaStream_t stream) {
    int device = 0, sms = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (n_ctas <= 0) n_ctas = sms;
    params.nloc_max = (params.n + n_ctas - 1) / n_ctas;
    if constexpr (MODE != CSG_ARITH_FP64) {
        // a ring has at most 2 max_degree + 1 vertices
        if (params.allow_dataflow && params.max_degree > 0 && 2 * params.max_degree + 1 <= kRingMax) {
            const size_t smem = sizeof(float3) * (threads / 32) * (32 / G) * kRingMax +
                                static_cast<size_t>(params.nloc_max) * sizeof(int) * (kRingMax + params.max_degree + 4) +
                                sizeof(int) * (2 * static_cast<size_t>(params.n_levels) + params.stride);
            if (smem <= kMaxTopologySmem) return launch_dataflow<MODE, G>(params, n_ctas, threads, smem, stream);
        }
    }
    const size_t smem = static_cast<size_t>(params.nloc_max) * (params.max_degree * sizeof(int4) + 2 * sizeof(int)) +
                        sizeof(int) * (2 * static_cast<size_t>(params.n_levels) + params.stride);
    if (params.max_degree > 0 && smem <= kMaxTopologySmem)
        return launch_variant<MODE, G, true>(params, n_ctas, threads, smem, stream);
    return launch_variant<MODE, G, false>(params, n_ctas, threads, 0, stream);
}

template <int MODE>
int dispatch_lanes(const ArealParams& params, int n_ctas, int threads, int lanes, cudaStream_t stream) {
    switch (lanes) {
        case 4: return launch<MODE, 4>(params, n_ctas, threads, stream);
        case 8: return launch<MODE, 8>(params, n_ctas, threads, stream);
        case 16: return launch<MODE, 16>(params, n_ctas, threads, stream);
        default: return csg::fail(CSG_ERR_ARG, "lanes_per_vertex must be 4, 8 or 16 (got %d)", lanes);
    }
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Barrier whose expected arrival count is one more than the grid holds: the
// bounded wait must give up and record CSG_ERR_TIMEOUT.
__global__ void k_div3_selftest(const double* __restrict__ x, long long n, double* __restrict__ a,
                                double* __restrict__ b) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = __ddiv_rn(x[i], 3.0);
    b[i] = csg::div3_rn(x[i]);
}

__global__ void barrier_timeout_selftest_kernel(csg::Control* ctl, unsigned long long timeout_ns) {
    unsigned int phase = 1;
    csg::grid_barrier(ctl, phase, timeout_ns, 1);
}

}  // namespace

extern "C" {

size_t csg_areal_scratch_bytes(int n_vertices, int arithmetic) {
    if (n_vertices < 1 || (arithmetic != CSG_ARITH_CAT && arithmetic != CSG_ARITH_FP32 && arithmetic != CSG_ARITH_FP64))
        return 0;
    // float64: a double4 working copy; float32 modes: four published 8-byte
    // words per vertex and four projected ones (the dataflow form; the barrier
    // form uses the first 16 bytes per vertex)
    return sizeof(csg::Control) + align256(64 * static_cast<size_t>(n_vertices));
}

int csg_areal_sweeps(void* points, int n_vertices, const int32_t* slot_off, const int32_t* slot_tri,
                     const int32_t* order, const int32_t* level_begin, const int32_t* level_end, int n_levels,
                     int level_stride, int max_degree, int iterations, int project_every, double radius, int arithmetic, void* scratch,
                     size_t scratch_bytes, int n_ctas, int threads_per_cta, int lanes_per_vertex, double timeout_s,
                     csg_stream_t stream) {
    if (!points || n_vertices < 1 || !slot_off || !slot_tri || !order || !level_begin || !level_end || !scratch)
        return csg::fail(CSG_ERR_ARG, "areal sweeps: null pointer or empty mesh");
    if (n_levels < 1 || n_levels > n_vertices || level_stride < 1 || iterations < 1 || project_every < 0 ||
        max_degree < 0)
        return csg::fail(CSG_ERR_ARG, "areal sweeps: bad schedule (levels %d, stride %d, iterations %d, project %d)",
                         n_levels, level_stride, iterations, project_every);
    {
        const long long sweeps_per_epoch = project_every > 0 ? project_every : iterations;
        if ((sweeps_per_epoch - 1) * static_cast<long long>(level_stride) + n_levels >= (1LL << 31))
            return csg::fail(CSG_ERR_ARG, "areal sweeps: wavefront epoch longer than 2^31 steps");
    }
    if (arithmetic < CSG_ARITH_CAT || arithmetic > CSG_ARITH_FP64)
        return csg::fail(CSG_ERR_ARG, "areal sweeps: unknown arithmetic %d", arithmetic);
    if (scratch_bytes < csg_areal_scratch_bytes(n_vertices, arithmetic))
        return csg::fail(CSG_ERR_ARG, "areal sweeps: scratch %zu bytes < required %zu", scratch_bytes,
                         csg_areal_scratch_bytes(n_vertices, arithmetic));
    if (reinterpret_cast<uintptr_t>(scratch) % 256 != 0 || reinterpret_cast<uintptr_t>(slot_tri) % 16 != 0)
        return csg::fail(CSG_ERR_ARG, "areal sweeps: scratch must be 256-byte and slot_tri 16-byte aligned");
    if (threads_per_cta <= 0) threads_per_cta = 512;
    if (lanes_per_vertex <= 0) lanes_per_vertex = 8;
    if (threads_per_cta % 32 != 0 || threads_per_cta > 512)
        return csg::fail(CSG_ERR_ARG, "areal sweeps: threads_per_cta must be a multiple of 32 up to 512");
    if (timeout_s <= 0.0) timeout_s = 2.0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    ArealParams p{};
    p.points = points;
    p.ctl = static_cast<csg::Control*>(scratch);
    p.work = static_cast<char*>(scratch) + sizeof(csg::Control);
    p.slot_tri = reinterpret_cast<const int4*>(slot_tri);
    p.slot_off = slot_off;
    p.order = order;
    p.level_begin = level_begin;
    p.level_end = level_end;
    p.n = n_vertices;
    p.n_levels = n_levels;
    p.stride = level_stride;
    p.max_degree = max_degree;
    p.iterations = iterations;
    p.project_every = project_every;
    p.allow_dataflow = 1;
    p.radius = radius;
    p.timeout_ns = static_cast<unsigned long long>(timeout_s * 1e9);
    CSG_CUDA_CHECK(cudaMemsetAsync(scratch, 0, sizeof(csg::Control), s));
    switch (arithmetic) {
        case CSG_ARITH_CAT: return dispatch_lanes<CSG_ARITH_CAT>(p, n_ctas, threads_per_cta, lanes_per_vertex, s);
        case CSG_ARITH_FP32: return dispatch_lanes<CSG_ARITH_FP32>(p, n_ctas, threads_per_cta, lanes_per_vertex, s);
        default: return dispatch_lanes<CSG_ARITH_FP64>(p, n_ctas, threads_per_cta, lanes_per_vertex, s);
    }
}

int csg_selftest_div3(const double* x, long long n, double* by_division, double* by_multiplies, csg_stream_t stream) {
    if (!x || n < 0 || !by_division || !by_multiplies) return csg::fail(CSG_ERR_ARG, "div3 self-test: bad arguments");
    if (n == 0) return CSG_OK;
    (csg::note_launch(), k_div3_selftest<<<static_cast<unsigned>((n + 255) / 256), 256, 0,
                                          reinterpret_cast<cudaStream_t>(stream)>>>(x, n, by_division, by_multiplies));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_selftest_barrier_timeout(void* scratch, size_t scratch_bytes, double timeout_s, csg_stream_t stream) {
    if (!scratch || scratch_bytes < sizeof(csg::Control) || timeout_s <= 0.0 || timeout_s > 10.0)
        return csg::fail(CSG_ERR_ARG, "barrier self-test: need 256 bytes of scratch and 0 < timeout_s <= 10");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    csg::Control* ctl = static_cast<csg::Control*>(scratch);
    unsigned long long timeout_ns = static_cast<unsigned long long>(timeout_s * 1e9);
    CSG_CUDA_CHECK(cudaMemsetAsync(scratch, 0, sizeof(csg::Control), s));
    void* args[] = {&ctl, &timeout_ns};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(barrier_timeout_selftest_kernel), dim3(2),
                                               dim3(32), args, 0, s));
    csg::note_launch();
    return CSG_OK;
}

int csg_read_status(const void* scratch, csg_stream_t stream, int* status, int* where) {
    if (!scratch || !status) return csg::fail(CSG_ERR_ARG, "read_status: null pointer");
    csg::Control ctl{};
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    CSG_CUDA_CHECK(cudaMemcpyAsync(&ctl, scratch, sizeof(ctl), cudaMemcpyDeviceToHost, s));
    CSG_CUDA_CHECK(cudaStreamSynchronize(s));
    *status = ctl.status;
    if (where) *where = ctl.where;
    return CSG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of csg_areal_sweeps.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA stream
// capture is active on its thread (cudaMalloc is refused in the default
// capture mode), hosts that hand all device memory to their own pool
// allocator up front, and thin foreign-function bindings that pass device
// pointers they were given but own no device allocator.  For them the sweep
// kernel's working memory (the 256-byte control block and the float4 /
// double4 position working copy) lives in the file-scope array below, which
// every GPU that loads this library holds until the process exits.
// Limits: 262,144 vertices in the float32 modes, 131,072 in float64 mode.

namespace {
constexpr size_t kNoAllocWorkBytes = static_cast<size_t>(262144) * sizeof(float4);  // 4 MiB
constexpr size_t kNoAllocBytes = sizeof(csg::Control) + kNoAllocWorkBytes;
}  // namespace

static __device__ __align__(256) unsigned char g_areal_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mutex;
constexpr int kNoAllocMaxDevices = 64;
void* g_noalloc_address[kNoAllocMaxDevices] = {};

// Device address of g_areal_noalloc_scratch on the current device, looked up
// once per device (the name itself is only a host-side stand-in).  The cached
// address belongs to the device's primary context: after cudaDeviceReset the
// module may load elsewhere, so this entry point must not be used across a
// device reset.
int noalloc_scratch(void** out) {
    int device = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    if (device < 0 || device >= kNoAllocMaxDevices)
        return csg::fail(CSG_ERR_UNSUPPORTED, "areal sweeps (no-alloc): device ordinal %d >= %d", device,
                         kNoAllocMaxDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_address[device] == nullptr) {
        void* address = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&address, g_areal_noalloc_scratch);
        if (err != cudaSuccess || address == nullptr)
            return csg::fail(CSG_ERR_CUDA, "areal sweeps (no-alloc): cudaGetSymbolAddress failed: %s",
                             cudaGetErrorString(err));
        g_noalloc_address[device] = address;
    }
    *out = g_noalloc_address[device];
    return CSG_OK;
}
}  // namespace

extern "C" int csg_areal_sweeps_noalloc(void* points, int n_vertices, const int32_t* slot_off, const int32_t* slot_tri,
                                        const int32_t* order, const int32_t* level_begin, const int32_t* level_end,
                                        int n_levels, int level_stride, int max_degree, int iterations,
                                        int project_every, double radius, int arithmetic, int n_ctas,
                                        int threads_per_cta, int lanes_per_vertex, double timeout_s,
                                        int* status_out, csg_stream_t stream) {
    if (!points || n_vertices < 1 || !slot_off || !slot_tri || !order || !level_begin || !level_end)
        return csg::fail(CSG_ERR_ARG, "areal sweeps (no-alloc): null pointer or empty mesh");
    if (arithmetic < CSG_ARITH_CAT || arithmetic > CSG_ARITH_FP64)
        return csg::fail(CSG_ERR_ARG, "areal sweeps (no-alloc): unknown arithmetic %d", arithmetic);
    // the barrier form: a float4 (float32 modes) or double4 working copy
    const size_t need = sizeof(csg::Control) +
                        align256((arithmetic == CSG_ARITH_FP64 ? sizeof(D4) : sizeof(float4)) *
                                 static_cast<size_t>(n_vertices));
    if (need > kNoAllocBytes)
        return csg::fail(CSG_ERR_ARG,
                         "areal sweeps (no-alloc): %d vertices need %zu bytes of working memory, more than the "
                         "built-in %zu (at most %d vertices in float32 modes, %d in float64 mode)",
                         n_vertices, need, kNoAllocBytes, 262144, 131072);
    if (n_levels < 1 || n_levels > n_vertices || level_stride < 1 || iterations < 1 || project_every < 0 ||
        max_degree < 0)
        return csg::fail(CSG_ERR_ARG, "areal sweeps (no-alloc): bad schedule (levels %d, stride %d, iterations %d)",
                         n_levels, level_stride, iterations);
    {
        const long long sweeps_per_epoch = project_every > 0 ? project_every : iterations;
        if ((sweeps_per_epoch - 1) * static_cast<long long>(level_stride) + n_levels >= (1LL << 31))
            return csg::fail(CSG_ERR_ARG, "areal sweeps (no-alloc): wavefront epoch longer than 2^31 steps");
    }
    if (reinterpret_cast<uintptr_t>(slot_tri) % 16 != 0)
        return csg::fail(CSG_ERR_ARG, "areal sweeps (no-alloc): slot_tri must be 16-byte aligned");
    if (threads_per_cta <= 0) threads_per_cta = 512;
    if (lanes_per_vertex <= 0) lanes_per_vertex = 8;
    if (threads_per_cta % 32 != 0 || threads_per_cta > 512)
        return csg::fail(CSG_ERR_ARG, "areal sweeps (no-alloc): threads_per_cta must be a multiple of 32 up to 512");
    if (timeout_s <= 0.0) timeout_s = 2.0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (status_out != nullptr) {
        // reading the status back waits for the kernel, which a stream being captured cannot do
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        CSG_CUDA_CHECK(cudaStreamIsCapturing(s, &capture));
        if (capture != cudaStreamCaptureStatusNone)
            return csg::fail(CSG_ERR_ARG, "areal sweeps (no-alloc): status_out must be NULL while the stream is "
                                          "being captured");
    }
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    ArealParams p{};
    p.points = points;
    p.ctl = static_cast<csg::Control*>(scratch);
    p.work = static_cast<char*>(scratch) + sizeof(csg::Control);
    p.slot_tri = reinterpret_cast<const int4*>(slot_tri);
    p.slot_off = slot_off;
    p.order = order;
    p.level_begin = level_begin;
    p.level_end = level_end;
    p.n = n_vertices;
    p.n_levels = n_levels;
    p.stride = level_stride;
    p.max_degree = max_degree;
    p.iterations = iterations;
    p.project_every = project_every;
    p.radius = radius;
    p.timeout_ns = static_cast<unsigned long long>(timeout_s * 1e9);
    // The array keeps the previous call's contents: the control block (barrier
    // counter and status) must start at zero; the working copy is fully
    // rewritten from `points` by the kernel itself.
    CSG_CUDA_CHECK(cudaMemsetAsync(scratch, 0, sizeof(csg::Control), s));
    switch (arithmetic) {
        case CSG_ARITH_CAT: rc = dispatch_lanes<CSG_ARITH_CAT>(p, n_ctas, threads_per_cta, lanes_per_vertex, s); break;
        case CSG_ARITH_FP32: rc = dispatch_lanes<CSG_ARITH_FP32>(p, n_ctas, threads_per_cta, lanes_per_vertex, s); break;
        default: rc = dispatch_lanes<CSG_ARITH_FP64>(p, n_ctas, threads_per_cta, lanes_per_vertex, s); break;
    }
    if (rc || status_out == nullptr) return rc;
    csg::Control ctl{};
    CSG_CUDA_CHECK(cudaMemcpyAsync(&ctl, scratch, sizeof(ctl), cudaMemcpyDeviceToHost, s));
    CSG_CUDA_CHECK(cudaStreamSynchronize(s));
    *status_out = ctl.status;
    if (ctl.status != CSG_OK)
        return csg::fail(ctl.status, "areal sweeps (no-alloc): kernel reported status %d at barrier %d", ctl.status,
                         ctl.where);
    return CSG_OK;
}
