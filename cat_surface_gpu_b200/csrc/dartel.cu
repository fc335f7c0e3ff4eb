// 2-D DARTEL on the spherical lat-lon sheet, batched, for sm_100a.
//
// Every kernel works on a batch of B independent grids of the same size
// (fields laid out [B][channels][ny][nx], contiguous).  Arithmetic follows
// the reference's torch path operation by operation
// (src/cat_surface_gpu/dartel_grid.py, surface_warp.py); this file is
// compiled with --fmad=false so each multiply and add rounds once, which
// makes float64 and float32 results bit-identical to a sequential
// restatement with the same association order.
//
// Boundary rule (dartel_grid.py:190-208): x periodic, y reflected with
// period 2 ny (ny == 1 collapses y to row 0).  Maps are one-based; Jacobians
// are stored (j00, j10, j01, j11).
//
// The host half of this file orchestrates dartel_step (dartel_grid.py:
// 1420-1616), the membrane full multigrid (1211-1417) and the whole solve
// (surface_warp.py:239-367) as launch sequences on one stream, so a caller
// can capture a complete solve in one CUDA graph.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/catsurf_b200.h"
#include "errors.h"
#include "pdl.cuh"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int wrap_x(int ix, int nx) {
    int r = ix % nx;
    return r < 0 ? r + nx : r;
}

__device__ __forceinline__ int reflect_y(int iy, int ny) {
    if (ny == 1) return 0;
    const int period = 2 * ny;
    int r = iy % period;
    if (r < 0) r += period;
    return r >= ny ? period - r - 1 : r;
}

// Bilinear stencil of dartel_grid.py:348-366 at (x, y) (zero-based).
template <typename T>
struct Stencil {
    int i22, i12, i21, i11;  // flat offsets inside one channel
    T dx1, dx2, dy1, dy2;
    __device__ __forceinline__ Stencil(T x, T y, int nx, int ny) {
        const T fx = floor(x), fy = floor(y);
        const int ix = static_cast<int>(fx), iy = static_cast<int>(fy);
        dx1 = x - static_cast<T>(ix);
        dy1 = y - static_cast<T>(iy);
        dx2 = T(1) - dx1;
        dy2 = T(1) - dy1;
        const int x0 = wrap_x(ix, nx), x1 = wrap_x(ix + 1, nx);
        const int y0 = reflect_y(iy, ny), y1 = reflect_y(iy + 1, ny);
        i22 = y0 * nx + x0;
        i12 = y0 * nx + x1;
        i21 = y1 * nx + x0;
        i11 = y1 * nx + x1;
    }
    __device__ __forceinline__ T interp(const T* f) const {
        return (f[i22] * dx2 + f[i12] * dx1) * dy2 + (f[i21] * dx2 + f[i11] * dx1) * dy1;
    }
};

template <typename T>
__device__ __forceinline__ T unwrap(T c, T c22, T period) {
    return c - floor((c - c22) / period + T(0.5)) * period;
}

struct Pt {
    int b, x, y, i;  // batch, column, row, flat index in a channel
};

__device__ __forceinline__ bool point(int nx, int ny, Pt& p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return false;
    p.b = blockIdx.y;
    p.i = i;
    p.x = i % nx;
    p.y = i / nx;
    return true;
}

// Neighbour offsets with the boundary rule.
__device__ __forceinline__ int nb(int x, int y, int dx, int dy, int nx, int ny) {
    return reflect_y(y + dy, ny) * nx + wrap_x(x + dx, nx);
}

// ---------------------------------------------------------------- kernels

// map = id + v * s (dartel_grid.py:655-675 / 1644-1645) and
// jac = jacobian_of_displacement(v, s) (624-652); either output may be null.
template <typename T>
__global__ void k_smalldef(const T* __restrict__ v, T* __restrict__ map, T* __restrict__ jac, int nx, int ny, T s,
                           T hs) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const T* vx = v + static_cast<size_t>(p.b) * 2 * P;
    const T* vy = vx + P;
    if (map) {
        T* m = map + static_cast<size_t>(p.b) * 2 * P;
        m[p.i] = static_cast<T>(p.x + 1) + vx[p.i] * s;
        m[P + p.i] = static_cast<T>(p.y + 1) + vy[p.i] * s;
    }
    if (jac) {
        const int xm = nb(p.x, p.y, -1, 0, nx, ny), xp = nb(p.x, p.y, 1, 0, nx, ny);
        const int ym = nb(p.x, p.y, 0, -1, nx, ny), yp = nb(p.x, p.y, 0, 1, nx, ny);
        T* j = jac + static_cast<size_t>(p.b) * 4 * P;
        j[p.i] = (vx[xm] * T(-1) + vx[xp]) * hs + T(1);
        j[P + p.i] = (vy[xm] * T(-1) + vy[xp]) * hs;
        j[2 * P + p.i] = (vx[ym] * T(-1) + vx[yp]) * hs;
        j[3 * P + p.i] = (vy[ym] * T(-1) + vy[yp]) * hs + T(1);
    }
}

// (c, jc) = (b o a, J_b(a) . J_a) (dartel_grid.py:407-507) at point p, with the
// stencil of a at p; jac pointers may be null.
template <typename T>
__device__ __forceinline__ void compose_at(const Stencil<T>& st, const T* __restrict__ a, const T* __restrict__ ja,
                                           const T* __restrict__ b, const T* __restrict__ jb, T* __restrict__ c,
                                           T* __restrict__ jc, int nx, int ny, const Pt& p) {
    const int P = nx * ny;
    const size_t o2 = static_cast<size_t>(p.b) * 2 * P, o4 = static_cast<size_t>(p.b) * 4 * P;
    const T* Bm = b + o2;
    T* C = c + o2;
#pragma unroll
    for (int ch = 0; ch < 2; ++ch) {
        const T* f = Bm + ch * P;
        const T period = static_cast<T>(ch == 0 ? nx : ny);
        const T c22 = f[st.i22] - T(1);
        const T c12 = unwrap(f[st.i12] - T(1), c22, period);
        const T c21 = unwrap(f[st.i21] - T(1), c22, period);
        const T c11 = unwrap(f[st.i11] - T(1), c22, period);
        C[ch * P + p.i] = (c22 * st.dx2 + c12 * st.dx1) * st.dy2 + (c21 * st.dx2 + c11 * st.dx1) * st.dy1 + T(1);
    }
    if (jc) {
        const T* JA = ja + o4;
        const T* JB = jb + o4;
        const T jb00 = st.interp(JB), jb01 = st.interp(JB + P), jb10 = st.interp(JB + 2 * P),
                jb11 = st.interp(JB + 3 * P);
        const T ja0 = JA[p.i], ja1 = JA[P + p.i], ja2 = JA[2 * P + p.i], ja3 = JA[3 * P + p.i];
        T* J = jc + o4;
        J[p.i] = jb00 * ja0 + jb10 * ja1;
        J[P + p.i] = jb01 * ja0 + jb11 * ja1;
        J[2 * P + p.i] = jb00 * ja2 + jb10 * ja3;
        J[3 * P + p.i] = jb01 * ja2 + jb11 * ja3;
    }
}

template <typename T>
__global__ void k_compose(const T* __restrict__ a, const T* __restrict__ ja, const T* __restrict__ b,
                          const T* __restrict__ jb, T* __restrict__ c, T* __restrict__ jc, int nx, int ny) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const T* A = a + static_cast<size_t>(p.b) * 2 * P;
    const Stencil<T> st(A[p.i] - T(1), A[P + p.i] - T(1), nx, ny);
    compose_at(st, a, ja, b, jb, c, jc, nx, ny, p);
}

// jac_div_smalldef (dartel_grid.py:678-720) at one point.
template <typename T>
__device__ __forceinline__ void jacdiv_at(const T* J, const T* vx, const T* vy, const Pt& p, int nx, int ny, T hs,
                                          T out[4]) {
    const int P = nx * ny;
    const int xm = nb(p.x, p.y, -1, 0, nx, ny), xp = nb(p.x, p.y, 1, 0, nx, ny);
    const int ym = nb(p.x, p.y, 0, -1, nx, ny), yp = nb(p.x, p.y, 0, 1, nx, ny);
    const T d00 = (vx[xm] * T(-1) + vx[xp]) * hs + T(1);
    const T d10 = (vy[xm] * T(-1) + vy[xp]) * hs;
    const T d01 = (vx[ym] * T(-1) + vx[yp]) * hs;
    const T d11 = (vy[ym] * T(-1) + vy[yp]) * hs + T(1);
    const T det = d00 * d11 - d01 * d10;
    const T i00 = d11 / det, i10 = -d10 / det, i01 = -d01 / det, i11 = d00 / det;
    const T o00 = J[p.i], o10 = J[P + p.i], o01 = J[2 * P + p.i], o11 = J[3 * P + p.i];
    out[0] = o00 * i00 + o01 * i10;
    out[1] = o10 * i00 + o11 * i10;
    out[2] = o00 * i01 + o01 * i11;
    out[3] = o10 * i01 + o11 * i11;
}

template <typename T>
__global__ void k_jacdiv(const T* __restrict__ jac, const T* __restrict__ v, T* __restrict__ out, int nx, int ny,
                         T hs) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const T* vx = v + static_cast<size_t>(p.b) * 2 * P;
    T r[4];
    jacdiv_at(jac + static_cast<size_t>(p.b) * 4 * P, vx, vx + P, p, nx, ny, hs, r);
    T* o = out + static_cast<size_t>(p.b) * 4 * P;
    for (int k = 0; k < 4; ++k) o[k * P + p.i] = r[k];
}

// Block-level deterministic sum; partial[b * gridDim.x + blockIdx.x].
template <typename T>
__device__ __forceinline__ void block_sum(T value, T* partial) {
    __shared__ T buf[kThreads];
    buf[threadIdx.x] = value;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) buf[threadIdx.x] = buf[threadIdx.x] + buf[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[static_cast<size_t>(blockIdx.y) * gridDim.x + blockIdx.x] = buf[0];
}

// initialise_objfun (dartel_grid.py:723-775), optionally preceded by
// jac_div_smalldef (dartel_step's use, 1497-1512 / 1546-1561).  weights may
// be null (all ones).  Writes rhs [2], hess [3] and the objective partials.
template <typename T, bool JACDIV>
__global__ void k_objfun(const T* __restrict__ source, const T* __restrict__ target, const T* __restrict__ map,
                         const T* __restrict__ jac, const T* __restrict__ v, const T* __restrict__ weights,
                         T* __restrict__ rhs, T* __restrict__ hess, T* __restrict__ partial, int nx, int ny, T hs) {
    csg::pdl_begin();
    Pt p;
    const bool ok = point(nx, ny, p);
    T contrib = T(0);
    if (ok) {
        const int P = nx * ny;
        const size_t o1 = static_cast<size_t>(p.b) * P;
        const T* src = source + o1;
        const T* M = map + 2 * o1;
        T J[4];
        if (JACDIV) {
            const T* vx = v + 2 * o1;
            jacdiv_at(jac + 4 * o1, vx, vx + P, p, nx, ny, hs, J);
        } else {
            const T* JJ = jac + 4 * o1;
            for (int k = 0; k < 4; ++k) J[k] = JJ[k * P + p.i];
        }
        const Stencil<T> st(M[p.i] - T(1), M[P + p.i] - T(1), nx, ny);
        const T k22 = src[st.i22], k12 = src[st.i12], k21 = src[st.i21], k11 = src[st.i11];
        const T sampled = (k22 * st.dx2 + k12 * st.dx1) * st.dy2 + (k21 * st.dx2 + k11 * st.dx1) * st.dy1;
        const T diff = sampled - target[o1 + p.i];
        const T ddx = (k11 - k21) * st.dy1 + (k12 - k22) * st.dy2;
        const T ddy = (k11 * st.dx1 + k21 * st.dx2) - (k12 * st.dx1 + k22 * st.dx2);
        const T gx = J[0] * ddx + J[1] * ddy;
        const T gy = J[2] * ddx + J[3] * ddy;
        const T w = weights ? weights[o1 + p.i] : T(1);
        T* H = hess + 3 * o1;
        T* R = rhs + 2 * o1;
        H[p.i] = gx * gx * w;
        H[P + p.i] = gy * gy * w;
        H[2 * P + p.i] = gx * gy * w;
        R[p.i] = gx * diff * w;
        R[P + p.i] = gy * diff * w;
        contrib = diff * diff * w;
    }
    if (partial) block_sum(contrib, partial);
}

// One scaling-and-squaring increment (dartel_grid.py:832-893; the fused
// form of dartel_triton.py:345-477) at point p: b_out = b + inc_b, a_out = a +
// inc_a, inc = inc_b (inc may be null).  Out of place (the gathers read b and
// a at other points).  st is the stencil of map at p.
template <typename T>
__device__ __forceinline__ void squaring_at(const Stencil<T>& st, const T* __restrict__ b, const T* __restrict__ a,
                                            const T* __restrict__ map, const T* __restrict__ jac,
                                            T* __restrict__ b_out, T* __restrict__ a_out, T* __restrict__ inc,
                                            int nx, int ny, const Pt& p) {
    const int P = nx * ny;
    const size_t o1 = static_cast<size_t>(p.b) * P;
    const T* J = jac + 4 * o1;
    const T* Bv = b + 2 * o1;
    const T* Av = a + 3 * o1;
    const T j00 = J[p.i], j10 = J[P + p.i], j01 = J[2 * P + p.i], j11 = J[3 * P + p.i];
    const T det = j00 * j11 - j01 * j10;
    const T sbx = st.interp(Bv), sby = st.interp(Bv + P);
    const T sa00 = st.interp(Av), sa11 = st.interp(Av + P), sa01 = st.interp(Av + 2 * P);
    const T ibx = det * (sbx * j00 + sby * j10);
    const T iby = det * (sbx * j01 + sby * j11);
    const T t1 = sa00 * j00 + sa01 * j10;
    const T t2 = sa01 * j00 + sa11 * j10;
    const T t3 = sa00 * j01 + sa01 * j11;
    const T t4 = sa01 * j01 + sa11 * j11;
    const T ia00 = det * (t1 * j00 + t2 * j10);
    const T ia11 = det * (t3 * j01 + t4 * j11);
    const T ia01 = det * (t1 * j01 + t2 * j11);
    T* BO = b_out + 2 * o1;
    T* AO = a_out + 3 * o1;
    BO[p.i] = Bv[p.i] + ibx;
    BO[P + p.i] = Bv[P + p.i] + iby;
    AO[p.i] = Av[p.i] + ia00;
    AO[P + p.i] = Av[P + p.i] + ia11;
    AO[2 * P + p.i] = Av[2 * P + p.i] + ia01;
    if (inc) {
        T* I = inc + 2 * o1;
        I[p.i] = ibx;
        I[P + p.i] = iby;
    }
}

template <typename T>
__global__ void k_squaring(const T* __restrict__ b, const T* __restrict__ a, const T* __restrict__ map,
                           const T* __restrict__ jac, T* __restrict__ b_out, T* __restrict__ a_out,
                           T* __restrict__ inc, int nx, int ny) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const T* M = map + static_cast<size_t>(p.b) * 2 * P;
    const Stencil<T> st(M[p.i] - T(1), M[P + p.i] - T(1), nx, ny);
    squaring_at(st, b, a, map, jac, b_out, a_out, inc, nx, ny, p);
}

// One squaring step followed by the composition of the map with itself, in one
// pass: (b, a) advance as in k_squaring and (map_out, jac_out) = (map o map,
// J(map) . J).  Both read the same map at the same stencil and neither reads
// what the other writes, so the pass equals the two launches; the increment
// k_squaring would store in map_out is overwritten by the composed map there.
template <typename T>
__global__ void k_squaring_compose(const T* __restrict__ b, const T* __restrict__ a, const T* __restrict__ map,
                                   const T* __restrict__ jac, T* __restrict__ b_out, T* __restrict__ a_out,
                                   T* __restrict__ map_out, T* __restrict__ jac_out, int nx, int ny) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const T* M = map + static_cast<size_t>(p.b) * 2 * P;
    const Stencil<T> st(M[p.i] - T(1), M[P + p.i] - T(1), nx, ny);
    squaring_at(st, b, a, map, jac, b_out, a_out, static_cast<T*>(nullptr), nx, ny, p);
    compose_at(st, map, jac, map, jac, map_out, jac_out, nx, ny, p);
}

// regularization_operator weights (dartel_grid.py:937-1015), host-computed
// in float64 exactly as the reference forms them, cast to T on use.
//   rtype 1: w00, w01, w10
//   rtype 0: wx0, wy0, wx1, wy1, wx2, wy2, wxy
//   rtype 2: w00, w01, w02, w10, w11, w20
struct RegWeights {
    double w[8];
};

RegWeights reg_weights(const double* params, int rtype) {
    const double sx = params[0], sy = params[1], mu = params[2], lam = params[3], id = params[4];
    const double sx2 = sx * sx, sy2 = sy * sy;
    RegWeights r{};
    if (rtype == 1) {
        r.w[0] = mu * (2.0 * sx2 + 2.0 * sy2) + id;
        r.w[1] = -mu * sy2;
        r.w[2] = -mu * sx2;
    } else if (rtype == 0) {
        r.w[0] = mu * (2.0 * sy2 + 4.0 * sx2) + 2.0 * lam * sx2 + id;
        r.w[1] = mu * (2.0 * sx2 + 4.0 * sy2) + 2.0 * lam * sy2 + id;
        r.w[2] = -(2.0 * mu + lam) * sx2;
        r.w[3] = -(2.0 * mu + lam) * sy2;
        r.w[4] = -mu * sx2;
        r.w[5] = -mu * sy2;
        r.w[6] = 0.25 * (lam + mu) * sx * sy;
    } else {
        const double sx4 = sx2 * sx2, sy4 = sy2 * sy2;
        r.w[0] = mu * (6.0 * sx4 + 6.0 * sy4 + 8.0 * sx2 * sy2) + id;
        r.w[1] = mu * (-4.0 * sx2 * sy2 - 4.0 * sy4);
        r.w[2] = mu * sy4;
        r.w[3] = mu * (-4.0 * sx4 - 4.0 * sx2 * sy2);
        r.w[4] = mu * (2.0 * sx2 * sy2);
        r.w[5] = mu * sx4;
    }
    return r;
}

// Membrane weights as relax_membrane / the Triton kernels form them
// (dartel_grid.py:1113-1116): w00 = mu (2 sx sx + 2 sy sy) + id.
struct MemWeights {
    double w00, w01, w10;
};

MemWeights mem_weights(const double* params) {
    const double sx = params[0], sy = params[1], mu = params[2], id = params[4];
    return {mu * (2.0 * sx * sx + 2.0 * sy * sy) + id, -mu * sy * sy, -mu * sx * sx};
}

template <typename T>
__device__ __forceinline__ void regularise_at(const T* vx, const T* vy, const Pt& p, int nx, int ny, int rtype,
                                              const RegWeights& rw, T out[2]) {
    auto at = [&](const T* f, int dx, int dy) { return f[nb(p.x, p.y, dx, dy, nx, ny)]; };
    const T* f[2] = {vx, vy};
    if (rtype == 1) {
        const T w00 = T(rw.w[0]), w01 = T(rw.w[1]), w10 = T(rw.w[2]);
        for (int c = 0; c < 2; ++c)
            out[c] = w00 * f[c][p.i] + w01 * (at(f[c], 0, -1) + at(f[c], 0, 1)) + w10 * (at(f[c], -1, 0) + at(f[c], 1, 0));
    } else if (rtype == 0) {
        const T wx0 = T(rw.w[0]), wy0 = T(rw.w[1]), wx1 = T(rw.w[2]), wy1 = T(rw.w[3]), wx2 = T(rw.w[4]),
                wy2 = T(rw.w[5]), wxy = T(rw.w[6]);
        const T cross_x = at(vy, -1, -1) - at(vy, -1, 1) - at(vy, 1, -1) + at(vy, 1, 1);
        const T cross_y = at(vx, -1, -1) - at(vx, -1, 1) - at(vx, 1, -1) + at(vx, 1, 1);
        out[0] = wx0 * vx[p.i] + wy2 * (at(vx, 0, -1) + at(vx, 0, 1)) + wx1 * (at(vx, -1, 0) + at(vx, 1, 0)) +
                 wxy * cross_x;
        out[1] = wy0 * vy[p.i] + wy1 * (at(vy, 0, -1) + at(vy, 0, 1)) + wx2 * (at(vy, -1, 0) + at(vy, 1, 0)) +
                 wxy * cross_y;
    } else {
        const T w00 = T(rw.w[0]), w01 = T(rw.w[1]), w02 = T(rw.w[2]), w10 = T(rw.w[3]), w11 = T(rw.w[4]),
                w20 = T(rw.w[5]);
        for (int c = 0; c < 2; ++c) {
            const T* g = f[c];
            out[c] = w00 * g[p.i] + w01 * (at(g, 0, -1) + at(g, 0, 1)) + w02 * (at(g, 0, -2) + at(g, 0, 2)) +
                     w10 * (at(g, -1, 0) + at(g, 1, 0)) +
                     w11 * (at(g, -1, -1) + at(g, 1, -1) + at(g, -1, 1) + at(g, 1, 1)) +
                     w20 * (at(g, -2, 0) + at(g, 2, 0));
        }
    }
}

template <typename T>
__global__ void k_regularise(const T* __restrict__ v, T* __restrict__ out, int nx, int ny, int rtype, RegWeights rw) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const T* vx = v + static_cast<size_t>(p.b) * 2 * P;
    T r[2];
    regularise_at(vx, vx + P, p, nx, ny, rtype, rw, r);
    T* o = out + static_cast<size_t>(p.b) * 2 * P;
    o[p.i] = r[0];
    o[P + p.i] = r[1];
}

// dartel_step's combination (dartel_grid.py:1575-1594):
//   code 1: rhs = (rhs_f - rhs_r) * s + reg(v), hess = (hess_f + hess_r) * s
//   code 0: rhs = rhs_f * s + reg(v),           hess = hess_f * s
// plus the partial sums of reg(v) . v and rhs . rhs (metrics).
template <typename T>
__global__ void k_combine(const T* __restrict__ rf, const T* __restrict__ rr, const T* __restrict__ hf,
                          const T* __restrict__ hr, const T* __restrict__ v, T* __restrict__ rhs, T* __restrict__ hess,
                          T* __restrict__ partial_reg, T* __restrict__ partial_norm, int nx, int ny, T s, RegWeights rw) {
    csg::pdl_begin();
    Pt p;
    const bool ok = point(nx, ny, p);
    T reg_dot = T(0), norm = T(0);
    if (ok) {
        const int P = nx * ny;
        const size_t o1 = static_cast<size_t>(p.b) * P;
        const T* vx = v + 2 * o1;
        T reg[2];
        regularise_at(vx, vx + P, p, nx, ny, 1, rw, reg);
        for (int c = 0; c < 2; ++c) {
            const T base = rr ? rf[2 * o1 + c * P + p.i] - rr[2 * o1 + c * P + p.i] : rf[2 * o1 + c * P + p.i];
            const T r = base * s + reg[c];
            rhs[2 * o1 + c * P + p.i] = r;
            norm = norm + r * r;
            reg_dot = reg_dot + reg[c] * vx[c * P + p.i];
        }
        for (int c = 0; c < 3; ++c) {
            const T base = hr ? hf[3 * o1 + c * P + p.i] + hr[3 * o1 + c * P + p.i] : hf[3 * o1 + c * P + p.i];
            hess[3 * o1 + c * P + p.i] = base * s;
        }
    }
    block_sum(reg_dot, partial_reg);
    block_sum(norm, partial_norm);
}

// (H + L_membrane) u (dartel_grid.py:1018-1070); with `b`, the residual b - (H + L) u.
// Flat offsets of a point's four neighbours under the boundary rule.
struct Nbr4 {
    int xm, xp, ym, yp;
};

__device__ __forceinline__ Nbr4 neighbours(int x, int y, int nx, int ny) {
    return {nb(x, y, -1, 0, nx, ny), nb(x, y, 1, 0, nx, ny), nb(x, y, 0, -1, nx, ny), nb(x, y, 0, 1, nx, ny)};
}

// membrane_apply_at (rtype 1) with the neighbour offsets given, for one batch element's fields.
template <typename T>
__device__ __forceinline__ void membrane_core(const T* __restrict__ H, const T* __restrict__ ux,
                                              const T* __restrict__ b, T* __restrict__ o, int P, int i, const Nbr4& n,
                                              const RegWeights& rw) {
    const T w00 = T(rw.w[0]), w01 = T(rw.w[1]), w10 = T(rw.w[2]);
    T reg[2];
    for (int c = 0; c < 2; ++c) {
        const T* f = ux + c * P;
        reg[c] = w00 * f[i] + w01 * (f[n.ym] + f[n.yp]) + w10 * (f[n.xm] + f[n.xp]);
    }
    const T u0 = ux[i], u1 = ux[P + i];
    const T a0 = reg[0] + H[i] * u0 + H[2 * P + i] * u1;
    const T a1 = reg[1] + H[2 * P + i] * u0 + H[P + i] * u1;
    o[i] = b[i] - a0;
    o[P + i] = b[P + i] - a1;
}

template <typename T>
__device__ __forceinline__ void membrane_apply_at(const T* __restrict__ hess, const T* __restrict__ u,
                                                  const T* __restrict__ b, T* __restrict__ out, int nx, int ny,
                                                  const RegWeights& rw, const Pt& p) {
    const int P = nx * ny;
    const size_t o1 = static_cast<size_t>(p.b) * P;
    const T* ux = u + 2 * o1;
    const T* H = hess + 3 * o1;
    T reg[2];
    regularise_at(ux, ux + P, p, nx, ny, 1, rw, reg);
    const T u0 = ux[p.i], u1 = ux[P + p.i];
    const T a0 = reg[0] + H[p.i] * u0 + H[2 * P + p.i] * u1;
    const T a1 = reg[1] + H[2 * P + p.i] * u0 + H[P + p.i] * u1;
    T* o = out + 2 * o1;
    if (b) {
        o[p.i] = b[2 * o1 + p.i] - a0;
        o[P + p.i] = b[2 * o1 + P + p.i] - a1;
    } else {
        o[p.i] = a0;
        o[P + p.i] = a1;
    }
}

template <typename T>
__global__ void k_membrane_apply(const T* __restrict__ hess, const T* __restrict__ u, const T* __restrict__ b,
                                 T* __restrict__ out, int nx, int ny, RegWeights rw) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    membrane_apply_at(hess, u, b, out, nx, ny, rw, p);
}

// One red-black half sweep, in place (dartel_grid.py:1187-1208 /
// dartel_triton.py:242-291): cells with ((x + y) & 1) == colour.  Exact for
// even nx and for nx == 1, where every neighbour read is either of the other
// colour or the cell itself.
// relax_at with the neighbour offsets given (o1: the batch element's point offset).
template <typename T>
__device__ __forceinline__ void relax_core(const T* __restrict__ hess, const T* __restrict__ b, T* __restrict__ u,
                                           int P, size_t o1, int i, const Nbr4& n, T w00, T w01, T w10) {
    T* ux = u + 2 * o1;
    T* uy = ux + P;
    const T rx = b[2 * o1 + i] - w01 * (ux[n.ym] + ux[n.yp]) - w10 * (ux[n.xm] + ux[n.xp]);
    const T ry = b[2 * o1 + P + i] - w01 * (uy[n.ym] + uy[n.yp]) - w10 * (uy[n.xm] + uy[n.xp]);
    const T* H = hess + 3 * o1;
    const T dxx = H[i] + w00;
    const T dyy = H[P + i] + w00;
    const T cr = H[2 * P + i];
    const T det = dxx * dyy * T(1.0000000001) - cr * cr;
    const T nxv = (dyy * rx - cr * ry) / det;
    const T nyv = (-cr * rx + dxx * ry) / det;
    ux[i] = nxv;
    uy[i] = nyv;
}

template <typename T>
__device__ __forceinline__ void relax_at(const T* __restrict__ hess, const T* __restrict__ b, T* __restrict__ u,
                                         int nx, int ny, T w00, T w01, T w10, const Pt& p) {
    const int P = nx * ny;
    relax_core(hess, b, u, P, static_cast<size_t>(p.b) * P, p.i, neighbours(p.x, p.y, nx, ny), w00, w01, w10);
}

template <typename T>
__global__ void k_relax(const T* __restrict__ hess, const T* __restrict__ b, T* __restrict__ u, int nx, int ny,
                        int colour, T w00, T w01, T w10) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    if (((p.x + p.y) & 1) != colour) return;
    relax_at(hess, b, u, nx, ny, w00, w01, w10, p);
}

// Direct 2x2 point solve of the coarsest level (dartel_grid.py:1318-1334).
template <typename T>
__global__ void k_point_solve(const T* __restrict__ hess, const T* __restrict__ b, T* __restrict__ u, int P, T id) {
    csg::pdl_begin();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const size_t o1 = static_cast<size_t>(blockIdx.y) * P;
    const T* H = hess + 3 * o1;
    const T dxx = H[i] + id, dyy = H[P + i] + id, cr = H[2 * P + i];
    const T det = dxx * dyy * T(1.0000000001) - cr * cr;
    const T b0 = b[2 * o1 + i], b1 = b[2 * o1 + P + i];
    u[2 * o1 + i] = (dyy * b0 - cr * b1) / det;
    u[2 * o1 + P + i] = (-cr * b0 + dxx * b1) / det;
}

template <typename T>
__device__ __forceinline__ T wt2(T d) {
    const T a = fabs(d);
    const T inner = T(0.75) - a * a;
    const T od = T(1.5) - a;
    const T outer = T(0.5) * od * od;
    return a < T(0.5) ? inner : (a < T(1.5) ? outer : T(0));
}

// Taps of resize_at along one axis for target index t: the three source offsets
// (rows: reflected and scaled by the source row length; columns: periodic) and the
// quadratic B-spline weights, formed as resize_at forms them.
template <typename T>
struct AxisTaps {
    int o[3];  // minus, centre, plus
    T w[3];
};

template <typename T>
__device__ __forceinline__ AxisTaps<T> row_taps(int y, int sny, int tny, int snx) {
    const T yl = (static_cast<T>(y) + T(0.5)) * static_cast<T>(sny) / static_cast<T>(tny) - T(0.5);
    const int yo = static_cast<int>(floor(yl + T(0.5)));
    const T yof = static_cast<T>(yo);
    AxisTaps<T> a;
    a.w[1] = wt2(yof - yl);
    a.w[0] = wt2(yof - T(1) - yl);
    a.w[2] = wt2(yof + T(1) - yl);
    a.o[0] = reflect_y(yo - 1, sny) * snx;
    a.o[1] = reflect_y(yo, sny) * snx;
    a.o[2] = reflect_y(yo + 1, sny) * snx;
    return a;
}

template <typename T>
__device__ __forceinline__ AxisTaps<T> col_taps(int x, int snx, int tnx) {
    const T xl = (static_cast<T>(x) + T(0.5)) * static_cast<T>(snx) / static_cast<T>(tnx) - T(0.5);
    const int xo = static_cast<int>(floor(xl + T(0.5)));
    const T xof = static_cast<T>(xo);
    AxisTaps<T> a;
    a.w[1] = wt2(xof - xl);
    a.w[0] = wt2(xof - T(1) - xl);
    a.w[2] = wt2(xof + T(1) - xl);
    a.o[0] = wrap_x(xo - 1, snx);
    a.o[1] = wrap_x(xo, snx);
    a.o[2] = wrap_x(xo + 1, snx);
    return a;
}

// One target value of the separable resize from its row and column taps (f: the source plane).
template <typename T>
__device__ __forceinline__ T resize_value(const T* __restrict__ f, const AxisTaps<T>& r, const AxisTaps<T>& c) {
    const T im = r.w[0] * f[r.o[0] + c.o[0]] + r.w[1] * f[r.o[1] + c.o[0]] + r.w[2] * f[r.o[2] + c.o[0]];
    const T ic = r.w[0] * f[r.o[0] + c.o[1]] + r.w[1] * f[r.o[1] + c.o[1]] + r.w[2] * f[r.o[2] + c.o[1]];
    const T ip = r.w[0] * f[r.o[0] + c.o[2]] + r.w[1] * f[r.o[1] + c.o[2]] + r.w[2] * f[r.o[2] + c.o[2]];
    return c.w[0] * im + c.w[1] * ic + c.w[2] * ip;
}

// Separable quadratic B-spline resize (dartel_grid.py:239-305), y pass then
// x pass, per target point; `accumulate` adds into dst (prolongation,
// dartel_grid.py:1380-1387).  Fields are [B * C][sny][snx] -> [B * C][tny][tnx].
template <typename T>
__device__ __forceinline__ void resize_at(const T* __restrict__ src, T* __restrict__ dst, int snx, int sny, int tnx,
                                          int tny, int accumulate, int plane, int i) {
    const int x = i % tnx, y = i / tnx;
    const T* f = src + static_cast<size_t>(plane) * snx * sny;
    const T r = resize_value(f, row_taps<T>(y, sny, tny, snx), col_taps<T>(x, snx, tnx));
    T* o = dst + static_cast<size_t>(plane) * tnx * tny;
    o[i] = accumulate ? o[i] + r : r;
}

template <typename T>
__global__ void k_resize(const T* __restrict__ src, T* __restrict__ dst, int snx, int sny, int tnx, int tny,
                         int accumulate) {
    csg::pdl_begin();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tnx * tny) return;
    resize_at(src, dst, snx, sny, tnx, tny, accumulate, static_cast<int>(blockIdx.y), i);
}

// ------------------------------------------------ fused coarse multigrid cycle
//
// The levels of a V-cycle at or below kCoarsePoints points per grid run as one
// launch with one CTA per batch element: the same per-point operations as the
// separate kernels (relax_at, membrane_apply_at, resize_at) in the same
// order, phases separated by __syncthreads.  A coarse level's work is a few
// thousand points, so one CTA covers it, and ~100 small launches per cycle
// become one.  Every level's Hessian, right-hand side, solution and residual
// live in shared memory for the whole cycle (at most ~1,100 points over all
// levels, 9 words each): the CTA reads the Hessians and the first level's
// right-hand side and solution once, and writes back the first level's
// solution, the only field read after the cycle.  Each point's neighbour
// offsets and each level pair's resize taps (per target row and column) are
// tabled once per launch, so the ~90 barrier-separated phases do no index or
// weight arithmetic (the values are the ones relax_at, membrane_apply_at and
// resize_at form).

constexpr int kCoarsePoints = 512;  // measured: 512 beats 0, 2048 and 8192 at 256 x 128
constexpr int kMaxLevels = 16;
constexpr int kCoarseThreads = 1024;
constexpr int kCoarseCycleThreads = 512;

template <typename T>
struct CoarseLevel {
    const T* A;  // Hessian [batch][3][ny][nx]
    T* B;        // right-hand side [batch][2][ny][nx]
    T* U;        // solution [batch][2][ny][nx]
    T* R;        // residual [batch][2][ny][nx]
    int nx, ny;
    T w00, w01, w10;
    RegWeights rw;
    int off;  // offset of the level's [A 3 | B 2 | U 2 | R 2] x nx x ny block in shared memory (elements)
};

template <typename T>
struct CoarseCycle {
    CoarseLevel<T> lv[kMaxLevels];
    int first, last, nit;
};

// Resize of one batch element's two planes with the target rows' and columns' taps tabled.
// The threads that work a phase of the coarse cycle and their barrier: the whole CTA,
// or (levels of at most 32 points) warp 0 alone with a warp barrier.
template <bool WARP>
struct Team {
    static __device__ __forceinline__ int rank() { return WARP ? (threadIdx.x & 31) : threadIdx.x; }
    static __device__ __forceinline__ int size() { return WARP ? 32 : blockDim.x; }
    static __device__ __forceinline__ void sync() {
        if (WARP) __syncwarp();
        else __syncthreads();
    }
};

// Resize of one batch element's two planes with the target rows' and columns' taps tabled.
template <bool WARP, typename T>
__device__ __forceinline__ void taps_resize(const T* src, int snx, int sny, T* dst, int tnx, int tny,
                                            const AxisTaps<T>* rows, const AxisTaps<T>* cols, int accumulate) {
    const int P = tnx * tny;
    for (int j = Team<WARP>::rank(); j < 2 * P; j += Team<WARP>::size()) {
        const int c = j >= P ? 1 : 0, i = j - c * P;
        const T r = resize_value(src + static_cast<size_t>(c) * snx * sny, rows[i / tnx], cols[i % tnx]);
        T* o = dst + static_cast<size_t>(c) * P;
        o[i] = accumulate ? o[i] + r : r;
    }
    Team<WARP>::sync();
}

// The shared-memory image of level L (one batch element, batch index 0).
template <typename T>
__device__ __forceinline__ CoarseLevel<T> shared_level(const CoarseLevel<T>& L, T* base) {
    CoarseLevel<T> S = L;
    const int P = L.nx * L.ny;
    T* a = base + L.off;
    S.A = a;
    S.B = a + 3 * P;
    S.U = a + 5 * P;
    S.R = a + 7 * P;
    return S;
}

// Red-black relaxation of a shared-memory level with tabled neighbour offsets.
template <bool WARP, typename T>
__device__ __forceinline__ void table_relax(const CoarseLevel<T>& L, const int4* tab, int nit) {
    const int P = L.nx * L.ny;
    for (int it = 0; it < 2 * nit; ++it) {
        const int colour = it % 2 == 0 ? 1 : 0;
        for (int i = Team<WARP>::rank(); i < P; i += Team<WARP>::size()) {
            const int4 t = tab[i];
            if (((i % L.nx + i / L.nx) & 1) == colour)
                relax_core(L.A, L.B, L.U, P, 0, i, Nbr4{t.x, t.y, t.z, t.w}, L.w00, L.w01, L.w10);
        }
        Team<WARP>::sync();
    }
}

// The down half of the V-cycle at level l: relaxation, residual, its restriction to
// level l + 1 and that level's zero solution.
template <bool WARP, typename T>
__device__ __forceinline__ void coarse_down(const CoarseCycle<T>& c, int l, T* base, const int4* tab,
                                            const AxisTaps<T>* rows, const AxisTaps<T>* cols) {
    const CoarseLevel<T> L = shared_level(c.lv[l], base);
    table_relax<WARP>(L, tab, c.nit);
    const int P = L.nx * L.ny;
    for (int i = Team<WARP>::rank(); i < P; i += Team<WARP>::size()) {
        const int4 t = tab[i];
        membrane_core(L.A, L.U, L.B, L.R, P, i, Nbr4{t.x, t.y, t.z, t.w}, L.rw);
    }
    Team<WARP>::sync();
    const CoarseLevel<T> N = shared_level(c.lv[l + 1], base);
    taps_resize<WARP>(L.R, L.nx, L.ny, N.B, N.nx, N.ny, rows, cols, 0);
    const int Pn = N.nx * N.ny;
    for (int j = Team<WARP>::rank(); j < 2 * Pn; j += Team<WARP>::size()) N.U[j] = T(0);
    Team<WARP>::sync();
}

// The up half at level l: prolongation of level l + 1's solution, then relaxation.
template <bool WARP, typename T>
__device__ __forceinline__ void coarse_up(const CoarseCycle<T>& c, int l, T* base, const int4* tab,
                                          const AxisTaps<T>* rows, const AxisTaps<T>* cols) {
    const CoarseLevel<T> L = shared_level(c.lv[l], base);
    const CoarseLevel<T> N = shared_level(c.lv[l + 1], base);
    taps_resize<WARP>(N.U, N.nx, N.ny, L.U, L.nx, L.ny, rows, cols, 1);
    table_relax<WARP>(L, tab, c.nit);
}

// cycle(first) of Fmg (host side) restricted to levels first..last, for batch element blockIdx.x.
template <typename T>
__global__ void __launch_bounds__(kCoarseCycleThreads) k_fmg_coarse_cycle(CoarseCycle<T> c) {
    csg::pdl_begin();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* base = reinterpret_cast<T*>(smem_raw);
    const int bi = blockIdx.x;
    int words = 0;
    for (int l = c.first; l <= c.last; ++l) {
        words += 9 * c.lv[l].nx * c.lv[l].ny;
    }
    // neighbour offsets of every point of every level, after the fields (16-byte aligned)
    int4* table = reinterpret_cast<int4*>(smem_raw + ((static_cast<size_t>(words) * sizeof(T) + 15) & ~size_t(15)));
    for (int l = c.first, toff = 0; l <= c.last; ++l) {
        const CoarseLevel<T>& L = c.lv[l];
        const CoarseLevel<T> S = shared_level(L, base);
        const int P = L.nx * L.ny;
        for (int j = threadIdx.x; j < 3 * P; j += blockDim.x)
            const_cast<T*>(S.A)[j] = L.A[3 * static_cast<size_t>(bi) * P + j];
        if (l == c.first)
            for (int j = threadIdx.x; j < 2 * P; j += blockDim.x) {
                S.B[j] = L.B[2 * static_cast<size_t>(bi) * P + j];
                S.U[j] = L.U[2 * static_cast<size_t>(bi) * P + j];
            }
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
            const Nbr4 n = neighbours(i % L.nx, i / L.nx, L.nx, L.ny);
            table[toff + i] = make_int4(n.xm, n.xp, n.ym, n.yp);
        }
        toff += P;
    }
    __syncthreads();
    int toff = 0;
    int level_toff[kMaxLevels];
    for (int l = c.first; l <= c.last; ++l) {
        level_toff[l] = toff;
        toff += c.lv[l].nx * c.lv[l].ny;
    }
    // resize taps per level pair: restriction rows/columns of level l + 1, prolongation rows/columns of l
    AxisTaps<T>* taps = reinterpret_cast<AxisTaps<T>*>(table + toff);
    int down_rows[kMaxLevels], down_cols[kMaxLevels], up_rows[kMaxLevels], up_cols[kMaxLevels];
    {
        int at = 0;
        for (int l = c.first; l < c.last; ++l) {
            const CoarseLevel<T>& L = c.lv[l];
            const CoarseLevel<T>& N = c.lv[l + 1];
            down_rows[l] = at;
            at += N.ny;
            down_cols[l] = at;
            at += N.nx;
            up_rows[l] = at;
            at += L.ny;
            up_cols[l] = at;
            at += L.nx;
            for (int k = threadIdx.x; k < N.ny + N.nx + L.ny + L.nx; k += blockDim.x) {
                AxisTaps<T> t;
                if (k < N.ny) t = row_taps<T>(k, L.ny, N.ny, L.nx);
                else if (k < N.ny + N.nx) t = col_taps<T>(k - N.ny, L.nx, N.nx);
                else if (k < N.ny + N.nx + L.ny) t = row_taps<T>(k - N.ny - N.nx, N.ny, L.ny, N.nx);
                else t = col_taps<T>(k - N.ny - N.nx - L.ny, N.nx, L.nx);
                taps[down_rows[l] + k] = t;
            }
        }
    }
    __syncthreads();
    // levels from `tail` on hold at most 32 points: warp 0 runs them with warp barriers
    int tail = c.last;
    while (tail > c.first && c.lv[tail - 1].nx * c.lv[tail - 1].ny <= 32) --tail;
    for (int l = c.first; l < tail; ++l)
        coarse_down<false>(c, l, base, table + level_toff[l], taps + down_rows[l], taps + down_cols[l]);
    if (threadIdx.x < 32) {
        for (int l = tail; l < c.last; ++l)
            coarse_down<true>(c, l, base, table + level_toff[l], taps + down_rows[l], taps + down_cols[l]);
        table_relax<true>(shared_level(c.lv[c.last], base), table + level_toff[c.last], c.nit);
        for (int l = c.last; l-- > tail;)
            coarse_up<true>(c, l, base, table + level_toff[l], taps + up_rows[l], taps + up_cols[l]);
    }
    __syncthreads();
    for (int l = tail; l-- > c.first;)
        coarse_up<false>(c, l, base, table + level_toff[l], taps + up_rows[l], taps + up_cols[l]);
    const CoarseLevel<T>& F = c.lv[c.first];
    const int P = F.nx * F.ny;
    const T* su = base + F.off + 5 * P;
    for (int j = threadIdx.x; j < 2 * P; j += blockDim.x) F.U[2 * static_cast<size_t>(bi) * P + j] = su[j];
}

// Shared memory of the coarse cycle over levels first..last (specs: (nx, ny) per level).
template <typename T>
size_t coarse_cycle_smem(const std::vector<std::pair<int, int>>& specs, size_t first) {
    size_t words = 0, points = 0;
    for (size_t l = first; l < specs.size(); ++l) {
        words += 9 * static_cast<size_t>(specs[l].first) * specs[l].second;
        points += static_cast<size_t>(specs[l].first) * specs[l].second;
    }
    size_t taps = 0;
    for (size_t l = first; l + 1 < specs.size(); ++l)
        taps += static_cast<size_t>(specs[l].first + specs[l].second + specs[l + 1].first + specs[l + 1].second);
    return ((words * sizeof(T) + 15) & ~size_t(15)) + points * sizeof(int4) + taps * sizeof(AxisTaps<T>);
}

// ------------------------------------------------ fused fine-level V-cycle legs
//
// On the fine levels (above kCoarsePoints points) one V-cycle leg used to be
// 2 nit red-black half-sweep launches plus a residual and a restriction
// launch going down, and a prolongation plus 2 nit half-sweeps going up.
// Here each leg of each level is one launch: a CTA copies its tile of the
// level and a halo into shared memory, runs all the leg's steps there and
// writes back its tile.  A red-black half-sweep reads only neighbours one
// step away, so after k half-sweeps the values are exact everywhere at
// least k cells inside the copied region (the true y edges reflect onto
// copied rows and x is periodic, so only the region's cut edges shrink);
// with a halo of 2 nit + 2 the tile and one ring round it hold exact
// residuals for the restriction taps.  Every point sees the same operands in
// the same order as in the separate kernels (relax_at, membrane_apply_at,
// resize_at), so results are bit-identical; halo points are recomputed by
// neighbouring tiles instead of exchanged.

constexpr int kTileX = 32, kTileY = 16;

struct TileGeom {
    int x0, x1, y0, y1;  // the tile's interior (global, half-open)
    int gx0, wx;         // copied columns: gx0 .. gx0 + wx - 1 (unwrapped), or all nx when full_x
    int gy0, wy;         // copied rows (clipped to the grid)
    bool full_x;
};

__device__ __forceinline__ TileGeom tile_geom(int nx, int ny, int halo) {
    const int tiles_x = (nx + kTileX - 1) / kTileX;
    TileGeom g;
    const int tx = static_cast<int>(blockIdx.x) % tiles_x, ty = static_cast<int>(blockIdx.x) / tiles_x;
    g.x0 = tx * kTileX;
    g.x1 = min(nx, g.x0 + kTileX);
    g.y0 = ty * kTileY;
    g.y1 = min(ny, g.y0 + kTileY);
    g.full_x = (g.x1 - g.x0) + 2 * halo >= nx;
    g.gx0 = g.full_x ? 0 : g.x0 - halo;
    g.wx = g.full_x ? nx : (g.x1 - g.x0) + 2 * halo;
    g.gy0 = max(0, g.y0 - halo);
    g.wy = min(ny, g.y1 + halo) - g.gy0;
    return g;
}

// Image coordinates of the x neighbour of image column ix (dx = -1 / +1).
__device__ __forceinline__ int image_x(const TileGeom& g, int ix, int dx, int nx) {
    return g.full_x ? wrap_x(ix + dx, nx) : ix + dx;
}
// Image row of the y neighbour of global row gy (reflected at the grid edges).
__device__ __forceinline__ int image_y(const TileGeom& g, int gy, int dy, int ny) {
    return reflect_y(gy + dy, ny) - g.gy0;
}

template <typename T>
struct FineImage {
    T* a;  // [3][wy][wx]
    T* b;  // [2][wy][wx]
    T* u;  // [2][wy][wx]
    int n;  // wx * wy
};

// Copy A, B and U of batch element bi over the tile's region into shared memory.
template <typename T>
__device__ void load_image(const T* __restrict__ A, const T* __restrict__ B, const T* __restrict__ U,
                           const TileGeom& g, int nx, int ny, int bi, FineImage<T>& im) {
    const int P = nx * ny;
    const size_t o1 = static_cast<size_t>(bi) * P;
    for (int q = threadIdx.x; q < im.n; q += blockDim.x) {
        const int ix = q % g.wx, iy = q / g.wx;
        const int gi = (g.gy0 + iy) * nx + wrap_x(g.gx0 + ix, nx);
        for (int c = 0; c < 3; ++c) im.a[c * im.n + q] = A[3 * o1 + c * P + gi];
        for (int c = 0; c < 2; ++c) {
            im.b[c * im.n + q] = B[2 * o1 + c * P + gi];
            im.u[c * im.n + q] = U[2 * o1 + c * P + gi];
        }
    }
}

// The points of one colour a thread owns in a leg: the r-th point of that
// colour in row-major image order for r = threadIdx.x + j * blockDim.x (an
// image row has an even width, so it holds wx / 2 points of each colour).
// Each carries its image index, its neighbours' image indices and its depth,
// the number of steps (each reading one cell away) after which it is still
// exact: its distance to the nearest cut edge of the region (x edges unless
// the region spans the periodic x range, y edges inside the grid); all are
// formed once per leg instead of once per half-sweep.
// measured on 2 maps x 256 x 128 float64: 512 threads with two points of each colour
// solve in 8.27 ms against 9.08 ms for 256 threads with three
constexpr int kLegPts = 2;
constexpr int kLegThreads = 512;

struct LegPoint {
    int q;  // image index, -1 for an empty slot
    int depth;
    int xm, xp, ym, yp;
};

__device__ __forceinline__ LegPoint leg_point(const TileGeom& g, int nx, int ny, int colour, int r) {
    LegPoint p{-1, 0, 0, 0, 0, 0};
    const int half = g.wx >> 1;
    if (r >= half * g.wy) return p;
    const int iy = r / half;
    const int ix = 2 * (r - iy * half) + ((colour - g.gx0 - g.gy0 - iy) & 1);
    p.q = iy * g.wx + ix;
    int d = 1 << 30;
    if (!g.full_x) d = min(d, min(ix, g.wx - 1 - ix));
    if (g.gy0 > 0) d = min(d, iy);
    if (g.gy0 + g.wy < ny) d = min(d, g.wy - 1 - iy);
    p.depth = d;
    if (d >= 1) {  // every neighbour lies inside the image
        const int gy = g.gy0 + iy;
        p.xm = iy * g.wx + image_x(g, ix, -1, nx);
        p.xp = iy * g.wx + image_x(g, ix, 1, nx);
        p.ym = image_y(g, gy, -1, ny) * g.wx + ix;
        p.yp = image_y(g, gy, 1, ny) * g.wx + ix;
    }
    return p;
}

struct LegPoints {
    LegPoint c[2][kLegPts];  // by colour
};

__device__ __forceinline__ void own_points(const TileGeom& g, int nx, int ny, LegPoints& own) {
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int j = 0; j < kLegPts; ++j) own.c[c][j] = leg_point(g, nx, ny, c, threadIdx.x + j * blockDim.x);
}

// relax_at on the image: one half-sweep of `colour` over the owned points exact after `k` steps.
template <int COLOUR, typename T>
__device__ __forceinline__ void image_half_sweep(FineImage<T>& im, const LegPoints& own, int k, T w00, T w01,
                                                 T w10) {
    T* ux = im.u;
    T* uy = im.u + im.n;
#pragma unroll
    for (int j = 0; j < kLegPts; ++j) {
        const LegPoint& p = own.c[COLOUR][j];
        if (p.q < 0 || p.depth < k) continue;
        const int q = p.q;
        const T rx = im.b[q] - w01 * (ux[p.ym] + ux[p.yp]) - w10 * (ux[p.xm] + ux[p.xp]);
        const T ry = im.b[im.n + q] - w01 * (uy[p.ym] + uy[p.yp]) - w10 * (uy[p.xm] + uy[p.xp]);
        const T dxx = im.a[q] + w00;
        const T dyy = im.a[im.n + q] + w00;
        const T cr = im.a[2 * im.n + q];
        const T det = dxx * dyy * T(1.0000000001) - cr * cr;
        const T nxv = (dyy * rx - cr * ry) / det;
        const T nyv = (-cr * rx + dxx * ry) / det;
        ux[q] = nxv;
        uy[q] = nyv;
    }
    __syncthreads();
}

// 2 nit half-sweeps, colour 1 first (the order of the separate relax launches).
template <typename T>
__device__ void image_relax(FineImage<T>& im, const LegPoints& own, int nit, T w00, T w01, T w10) {
    for (int it = 0; it < nit; ++it) {
        image_half_sweep<1>(im, own, 2 * it + 1, w00, w01, w10);
        image_half_sweep<0>(im, own, 2 * it + 2, w00, w01, w10);
    }
}

template <typename T>
__device__ void store_tile(const FineImage<T>& im, const TileGeom& g, int nx, int ny, int bi, T* __restrict__ U) {
    const int P = nx * ny;
    const size_t o1 = static_cast<size_t>(bi) * P;
    const int tw = g.x1 - g.x0, th = g.y1 - g.y0;
    for (int q = threadIdx.x; q < tw * th; q += blockDim.x) {
        const int gx = g.x0 + q % tw, gy = g.y0 + q / tw;
        const int iq = (gy - g.gy0) * g.wx + (g.full_x ? gx : gx - g.gx0);
        U[2 * o1 + gy * nx + gx] = im.u[iq];
        U[2 * o1 + P + gy * nx + gx] = im.u[im.n + iq];
    }
}

// A leg reads the level's solution from Uin and writes its tiles to Uout, a
// different buffer: tiles of one launch read each other's halos, so none may
// overwrite what another still reads (down: U -> the level's R buffer; up:
// R -> U).
template <typename T>
struct FineLeg {
    const T* A;    // this level's Hessian [batch][3][ny][nx]
    const T* B;    // right-hand side [batch][2][ny][nx]
    const T* Uin;  // solution before the leg [batch][2][ny][nx]
    T* Uout;       // solution after the leg
    int nx, ny;
    T w00, w01, w10;
    RegWeights rw;
    T* nB;  // down: the next coarser level's right-hand side (restricted residual)
    T* nU;  // down: the next coarser level's solution (zeroed); up: the coarser solution to prolongate
    int cnx, cny;
    int nit;
};

// Down leg of level l: 2 nit half-sweeps, the residual b - (H + L) u and its
// restriction to level l + 1, whose solution is zeroed.  Halo 2 nit + 2.
template <typename T>
__global__ void __launch_bounds__(kLegThreads) k_vcycle_down(FineLeg<T> L) {
    csg::pdl_begin();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int bi = blockIdx.y;
    const TileGeom g = tile_geom(L.nx, L.ny, 2 * L.nit + 2);
    FineImage<T> im;
    im.n = g.wx * g.wy;
    im.a = reinterpret_cast<T*>(smem_raw);
    im.b = im.a + 3 * im.n;
    im.u = im.b + 2 * im.n;
    T* r = im.u + 2 * im.n;  // residual [2][wy][wx]
    LegPoints own;
    own_points(g, L.nx, L.ny, own);
    load_image(L.A, L.B, L.Uin, g, L.nx, L.ny, bi, im);
    __syncthreads();
    image_relax(im, own, L.nit, L.w00, L.w01, L.w10);
    // residual (membrane_apply_at on the image) where it is exact
    const int kr = 2 * L.nit + 1;
    const T w00 = T(L.rw.w[0]), w01 = T(L.rw.w[1]), w10 = T(L.rw.w[2]);
#pragma unroll
    for (int colour = 0; colour < 2; ++colour)
#pragma unroll
        for (int j = 0; j < kLegPts; ++j) {
            const LegPoint& p = own.c[colour][j];
            if (p.q < 0 || p.depth < kr) continue;
            const int q = p.q;
            T reg[2];
            for (int c = 0; c < 2; ++c) {
                const T* f = im.u + c * im.n;
                reg[c] = w00 * f[q] + w01 * (f[p.ym] + f[p.yp]) + w10 * (f[p.xm] + f[p.xp]);
            }
            const T u0 = im.u[q], u1 = im.u[im.n + q];
            const T a0 = reg[0] + im.a[q] * u0 + im.a[2 * im.n + q] * u1;
            const T a1 = reg[1] + im.a[2 * im.n + q] * u0 + im.a[im.n + q] * u1;
            r[q] = im.b[q] - a0;
            r[im.n + q] = im.b[im.n + q] - a1;
        }
    __syncthreads();
    store_tile(im, g, L.nx, L.ny, bi, L.Uout);
    // restriction (resize_at) of the residual to the coarse points whose centre tap lies in this tile
    const int snx = L.nx, sny = L.ny, tnx = L.cnx, tny = L.cny;
    const int X0 = max(0, (g.x0 - 2) * tnx / snx - 1), X1 = min(tnx, (g.x1 + 2) * tnx / snx + 2);
    const int Y0 = max(0, (g.y0 - 2) * tny / sny - 1), Y1 = min(tny, (g.y1 + 2) * tny / sny + 2);
    const int cw = X1 - X0, ch = Y1 - Y0;
    const size_t cP = static_cast<size_t>(tnx) * tny;
    for (int q = threadIdx.x; q < cw * ch; q += blockDim.x) {
        const int X = X0 + q % cw, Y = Y0 + q / cw;
        const T yl = (static_cast<T>(Y) + T(0.5)) * static_cast<T>(sny) / static_cast<T>(tny) - T(0.5);
        const int yo = static_cast<int>(floor(yl + T(0.5)));
        const T xl = (static_cast<T>(X) + T(0.5)) * static_cast<T>(snx) / static_cast<T>(tnx) - T(0.5);
        const int xo = static_cast<int>(floor(xl + T(0.5)));
        const int oy = reflect_y(yo, sny), ox = wrap_x(xo, snx);
        if (oy < g.y0 || oy >= g.y1 || ox < g.x0 || ox >= g.x1) continue;  // another tile's coarse point
        const T yof = static_cast<T>(yo);
        const T yw = wt2(yof - yl), ywm = wt2(yof - T(1) - yl), ywp = wt2(yof + T(1) - yl);
        const T xof = static_cast<T>(xo);
        const T xw = wt2(xof - xl), xwm = wt2(xof - T(1) - xl), xwp = wt2(xof + T(1) - xl);
        const int rm = (reflect_y(yo - 1, sny) - g.gy0) * g.wx, rc = (reflect_y(yo, sny) - g.gy0) * g.wx,
                  rp = (reflect_y(yo + 1, sny) - g.gy0) * g.wx;
        auto col = [&](int x) { return g.full_x ? wrap_x(x, snx) : wrap_x(x - g.gx0, snx); };
        const int cm = col(xo - 1), cc = col(xo), cp = col(xo + 1);
        for (int c = 0; c < 2; ++c) {
            const T* f = r + c * im.n;
            const T vm = ywm * f[rm + cm] + yw * f[rc + cm] + ywp * f[rp + cm];
            const T vc = ywm * f[rm + cc] + yw * f[rc + cc] + ywp * f[rp + cc];
            const T vp = ywm * f[rm + cp] + yw * f[rc + cp] + ywp * f[rp + cp];
            const size_t o = (2 * static_cast<size_t>(bi) + c) * cP + static_cast<size_t>(Y) * tnx + X;
            L.nB[o] = xwm * vm + xw * vc + xwp * vp;
            L.nU[o] = T(0);
        }
    }
}

// Up leg of level l: u += prolongation of the coarser solution (resize_at,
// accumulate), then 2 nit half-sweeps.  Halo 2 nit.
template <typename T>
__global__ void __launch_bounds__(kLegThreads) k_vcycle_up(FineLeg<T> L) {
    csg::pdl_begin();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int bi = blockIdx.y;
    const TileGeom g = tile_geom(L.nx, L.ny, 2 * L.nit);
    FineImage<T> im;
    im.n = g.wx * g.wy;
    im.a = reinterpret_cast<T*>(smem_raw);
    im.b = im.a + 3 * im.n;
    im.u = im.b + 2 * im.n;
    LegPoints own;
    own_points(g, L.nx, L.ny, own);
    load_image(L.A, L.B, L.Uin, g, L.nx, L.ny, bi, im);
    for (int q = threadIdx.x; q < im.n; q += blockDim.x) {
        const int ix = q % g.wx, iy = q / g.wx;
        const int x = wrap_x(g.gx0 + ix, L.nx), y = g.gy0 + iy;
        // resize_at's taps and weights for this point (the same for both channels)
        const T yl = (static_cast<T>(y) + T(0.5)) * static_cast<T>(L.cny) / static_cast<T>(L.ny) - T(0.5);
        const int yo = static_cast<int>(floor(yl + T(0.5)));
        const T yof = static_cast<T>(yo);
        const T yw = wt2(yof - yl), ywm = wt2(yof - T(1) - yl), ywp = wt2(yof + T(1) - yl);
        const int rm = reflect_y(yo - 1, L.cny) * L.cnx, rc = reflect_y(yo, L.cny) * L.cnx,
                  rp = reflect_y(yo + 1, L.cny) * L.cnx;
        const T xl = (static_cast<T>(x) + T(0.5)) * static_cast<T>(L.cnx) / static_cast<T>(L.nx) - T(0.5);
        const int xo = static_cast<int>(floor(xl + T(0.5)));
        const T xof = static_cast<T>(xo);
        const T xw = wt2(xof - xl), xwm = wt2(xof - T(1) - xl), xwp = wt2(xof + T(1) - xl);
        const int cm = wrap_x(xo - 1, L.cnx), cc = wrap_x(xo, L.cnx), cp = wrap_x(xo + 1, L.cnx);
        for (int c = 0; c < 2; ++c) {
            const T* src = L.nU + static_cast<size_t>(2 * bi + c) * L.cnx * L.cny;
            const T vm = ywm * src[rm + cm] + yw * src[rc + cm] + ywp * src[rp + cm];
            const T vc = ywm * src[rm + cc] + yw * src[rc + cc] + ywp * src[rp + cc];
            const T vp = ywm * src[rm + cp] + yw * src[rc + cp] + ywp * src[rp + cp];
            const T v = xwm * vm + xw * vc + xwp * vp;
            im.u[c * im.n + q] = im.u[c * im.n + q] + v;
        }
    }
    __syncthreads();
    image_relax(im, own, L.nit, L.w00, L.w01, L.w10);
    store_tile(im, g, L.nx, L.ny, bi, L.Uout);
}

// Points of the largest tile region of a level (tile plus halo, clipped to the grid).
inline size_t leg_points(int nx, int ny, int halo) {
    const int tw = std::min(kTileX, nx), th = std::min(kTileY, ny);
    const int wx = tw + 2 * halo >= nx ? nx : tw + 2 * halo;
    const int wy = std::min(ny, th + 2 * halo);
    return static_cast<size_t>(wx) * wy;
}

// Shared memory of one leg launch: A, B, U (+ the residual going down) over the largest tile region.
template <typename T>
size_t leg_smem(int nx, int ny, int halo, bool down) {
    return leg_points(nx, ny, halo) * (down ? 9 : 7) * sizeof(T);
}

constexpr size_t kLegSmemMax = 200 * 1024;
// Fused legs recompute their halos: past this many CTAs per level launch (tiles x
// batch) the separate launches are faster.  Measured on 256 x 128 sheets: in
// float64 a batch of 16 solves in 30.0 ms with the level-0 legs separate against
// 36.7 ms all fused (32.3 ms all separate); in float32 all fused is fastest.
template <typename T>
constexpr long long leg_max_ctas() {
    return sizeof(T) == 8 ? 256 : 1024;
}

// The restriction chain of a level-l field to every coarser level at or below
// kChainPoints points per grid, in one launch with one CTA per batch element:
// the same resize_at per point as separate k_resize launches, level after
// level, with __syncthreads between levels.  Each restricted level is kept in
// shared memory (at most ~700 points x channels over all levels) as the
// source of the next one, and written to its field.
constexpr int kChainPoints = 512;  // measured: 512 beats 2,048 (7.96 vs 8.14 ms per 256 x 128 solve) and matches 128

template <typename T>
struct ResizeChain {
    T* field[kMaxLevels];  // [batch * channels][ny][nx] per level
    int nx[kMaxLevels], ny[kMaxLevels];
    int off[kMaxLevels];   // offset of level l's [channels][ny][nx] image in shared memory (elements)
    int first, last, channels;
};

template <typename T>
__global__ void __launch_bounds__(kCoarseThreads) k_resize_chain(ResizeChain<T> c) {
    csg::pdl_begin();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* base = reinterpret_cast<T*>(smem_raw);
    const int bi = blockIdx.x;
    // every level's row and column taps first (after the level images), then the levels
    int words = 0, ntaps = 0;
    for (int l = c.first; l <= c.last; ++l) {
        words += c.channels * c.nx[l] * c.ny[l];
        ntaps += c.nx[l] + c.ny[l];
    }
    AxisTaps<T>* taps = reinterpret_cast<AxisTaps<T>*>(smem_raw + ((static_cast<size_t>(words) * sizeof(T) + 15) & ~size_t(15)));
    for (int l = c.first, at = 0; l <= c.last; ++l) {
        for (int k = threadIdx.x; k < c.ny[l] + c.nx[l]; k += blockDim.x)
            taps[at + k] = k < c.ny[l] ? row_taps<T>(k, c.ny[l - 1], c.ny[l], c.nx[l - 1])
                                       : col_taps<T>(k - c.ny[l], c.nx[l - 1], c.nx[l]);
        at += c.ny[l] + c.nx[l];
    }
    __syncthreads();
    for (int l = c.first, at = 0; l <= c.last; ++l) {
        const int P = c.nx[l] * c.ny[l];
        const size_t plane0 = static_cast<size_t>(c.channels) * bi;
        T* image = base + c.off[l];
        T* out = c.field[l] + plane0 * P;
        const T* src = l == c.first ? c.field[l - 1] + plane0 * c.nx[l - 1] * c.ny[l - 1] : base + c.off[l - 1];
        const AxisTaps<T>* rows = taps + at;
        const AxisTaps<T>* cols = rows + c.ny[l];
        for (int j = threadIdx.x; j < c.channels * P; j += blockDim.x) {
            const int ch = j / P, i = j - ch * P;
            const T r = resize_value(src + static_cast<size_t>(ch) * c.nx[l - 1] * c.ny[l - 1], rows[i / c.nx[l]],
                                     cols[i % c.nx[l]]);
            out[j] = r;
            image[j] = r;
        }
        at += c.ny[l] + c.nx[l];
        __syncthreads();
    }
}

template <typename T>
size_t resize_chain_smem(const ResizeChain<T>& c) {
    size_t words = 0, taps = 0;
    for (int l = c.first; l <= c.last; ++l) {
        words += static_cast<size_t>(c.channels) * c.nx[l] * c.ny[l];
        taps += static_cast<size_t>(c.nx[l] + c.ny[l]);
    }
    return ((words * sizeof(T) + 15) & ~size_t(15)) + taps * sizeof(AxisTaps<T>);
}

// Opt the leg, coarse-cycle and chain kernels in to more than 48 KB of dynamic
// shared memory, once per type and device (the first solve on a device runs eagerly, before any capture).
template <typename T>
void allow_big_smem() {
    static std::atomic<unsigned long long> done{0};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return;
    const unsigned long long bit = 1ULL << device;
    if (done.load() & bit) return;
    cudaFuncSetAttribute(reinterpret_cast<const void*>(k_vcycle_down<T>), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kLegSmemMax));
    cudaFuncSetAttribute(reinterpret_cast<const void*>(k_vcycle_up<T>), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kLegSmemMax));
    cudaFuncSetAttribute(reinterpret_cast<const void*>(k_fmg_coarse_cycle<T>),
                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kLegSmemMax));
    cudaFuncSetAttribute(reinterpret_cast<const void*>(k_resize_chain<T>), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kLegSmemMax));
    done.fetch_or(bit);
}

template <typename T>
__global__ void k_sub(T* __restrict__ v, const T* __restrict__ u, size_t n) {
    csg::pdl_begin();
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) v[i] = v[i] - u[i];
}

template <typename T>
__global__ void k_any_nonzero(const T* __restrict__ u, size_t n, int* flag) {
    csg::pdl_begin();
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n && u[i] != T(0)) atomicOr(flag, 1);
}

// Fixed-order reduction of per-block partials into metrics[b * stride + slot]
// (objective = forward + reverse partials; reg * 0.5; sqrt(norm)).
template <typename T>
__global__ void k_metrics(const T* __restrict__ obj_f, const T* __restrict__ obj_r, const T* __restrict__ reg,
                          const T* __restrict__ norm, int nblocks, T* __restrict__ metrics, int metric_stride) {
    csg::pdl_begin();
    const int b = blockIdx.x;
    if (threadIdx.x != 0) return;
    T of = T(0), orv = T(0), rg = T(0), nm = T(0);
    for (int k = 0; k < nblocks; ++k) {
        of = of + obj_f[static_cast<size_t>(b) * nblocks + k];
        if (obj_r) orv = orv + obj_r[static_cast<size_t>(b) * nblocks + k];
        rg = rg + reg[static_cast<size_t>(b) * nblocks + k];
        nm = nm + norm[static_cast<size_t>(b) * nblocks + k];
    }
    T* m = metrics + static_cast<size_t>(b) * metric_stride;
    m[0] = obj_r ? T(0.5) * of + T(0.5) * orv : T(0.5) * of;
    m[1] = rg * T(0.5);
    m[2] = sqrt(nm);
}

template <typename T>
__global__ void k_objective_out(const T* __restrict__ partial, int nblocks, T* __restrict__ out) {
    csg::pdl_begin();
    if (threadIdx.x != 0) return;
    T s = T(0);
    for (int k = 0; k < nblocks; ++k) s = s + partial[static_cast<size_t>(blockIdx.x) * nblocks + k];
    out[blockIdx.x] = T(0.5) * s;
}

// ------------------------------------------------------------- host side

struct Arena {
    char* base;
    size_t size;
    size_t used = 0;
    bool ok = true;
    template <typename T>
    T* take(size_t count) {
        const size_t bytes = (count * sizeof(T) + 255) & ~static_cast<size_t>(255);
        if (used + bytes > size) {
            ok = false;
            return nullptr;
        }
        T* p = reinterpret_cast<T*>(base ? base + used : nullptr);
        used += bytes;
        return p;
    }
};

inline dim3 grid_for(int points, int batch) { return dim3((points + kThreads - 1) / kThreads, batch); }

std::vector<std::pair<int, int>> grid_levels(int nx, int ny) {
    std::vector<std::pair<int, int>> specs{{nx, ny}};
    while (specs.back().first >= 2 || specs.back().second >= 2) {
        const auto prev = specs.back();
        const std::pair<int, int> coarse{(prev.first + 1) / 2, (prev.second + 1) / 2};
        specs.push_back(coarse);
        if (coarse.first < 2 && coarse.second < 2) break;
    }
    return specs;
}

bool relax_supported(int nx) { return nx % 2 == 0 || nx == 1; }

// Multigrid workspace for one (batch, nx, ny).
template <typename T>
struct FmgBuffers {
    std::vector<std::pair<int, int>> specs;
    std::vector<T*> A, B, B0, U, R;
    int* flag = nullptr;
    bool carve(Arena& ar, int batch, int nx, int ny) {
        specs = grid_levels(nx, ny);
        const size_t L = specs.size();
        A.assign(L, nullptr);
        B.assign(L, nullptr);
        B0.assign(L, nullptr);
        U.assign(L, nullptr);
        R.assign(L, nullptr);
        for (size_t l = 0; l < L; ++l) {
            const size_t P = static_cast<size_t>(specs[l].first) * specs[l].second;
            if (l > 0) {
                A[l] = ar.take<T>(3 * P * batch);
                B[l] = ar.take<T>(2 * P * batch);
                B0[l] = ar.take<T>(2 * P * batch);
                U[l] = ar.take<T>(2 * P * batch);
            }
            R[l] = ar.take<T>(2 * P * batch);
        }
        flag = ar.take<int>(1);
        return ar.ok;
    }
};

template <typename T>
struct Fmg {
    FmgBuffers<T>& buf;
    int batch;
    double base[5];
    int cycles, nit;
    cudaStream_t s;
    int nx0, ny0;

    void params_at(size_t l, double out[5]) const {
        out[0] = base[0] * buf.specs[l].first / nx0;
        out[1] = base[1] * buf.specs[l].second / ny0;
        out[2] = base[2];
        out[3] = base[3];
        out[4] = base[4];
    }
    void relax(size_t l) {
        const int nx = buf.specs[l].first, ny = buf.specs[l].second;
        double pr[5];
        params_at(l, pr);
        const MemWeights w = mem_weights(pr);
        for (int it = 0; it < 2 * nit; ++it)
            (csg::note_launch(), csg::launch_pdl(k_relax<T>, grid_for(nx * ny, batch), kThreads, 0, s, buf.A[l], buf.B[l], buf.U[l], nx, ny,
                                                                      it % 2 == 0 ? 1 : 0, T(w.w00), T(w.w01), T(w.w10)));
    }
    void resize(const T* src, size_t from, T* dst, size_t to, int channels, bool accumulate) {
        const auto f = buf.specs[from], t = buf.specs[to];
        (csg::note_launch(), csg::launch_pdl(k_resize<T>, grid_for(t.first * t.second, batch * channels), kThreads, 0, s, src, dst, f.first, f.second,
                                                                                     t.first, t.second, accumulate));
    }
    // First level of the fused coarse part: the finest level of at most
    // kCoarsePoints points (the whole cycle when the finest level is small).
    size_t coarse_first() const {
        size_t l = 0;
        while (l + 1 < buf.specs.size() &&
               static_cast<long long>(buf.specs[l].first) * buf.specs[l].second > kCoarsePoints)
            ++l;
        return l;
    }
    void coarse_cycle(size_t first) {
        const size_t last = buf.specs.size() - 1;
        CoarseCycle<T> c{};
        c.first = static_cast<int>(first);
        c.last = static_cast<int>(last);
        c.nit = nit;
        int off = 0;
        for (size_t l = first; l <= last; ++l) {
            double pr[5];
            params_at(l, pr);
            const MemWeights w = mem_weights(pr);
            c.lv[l] = CoarseLevel<T>{buf.A[l], buf.B[l], buf.U[l], buf.R[l], buf.specs[l].first, buf.specs[l].second,
                                     T(w.w00), T(w.w01), T(w.w10), reg_weights(pr, 1), off};
            off += 9 * buf.specs[l].first * buf.specs[l].second;
        }
        allow_big_smem<T>();
        (csg::note_launch(), csg::launch_pdl(k_fmg_coarse_cycle<T>, batch, kCoarseCycleThreads,
                                             coarse_cycle_smem<T>(buf.specs, first), s, c));
    }
    // One launch per fine leg (k_vcycle_down / k_vcycle_up) when every fine
    // level has an even x size and the tile regions fit in shared memory.
    // Level l runs as one down and one up leg launch when its tile regions fit the
    // shared memory and the per-thread point slots, and its tiles over the batch
    // stay within kLegMaxCtas CTAs (beyond that the halo recomputation costs more
    // than the separate launches save).
    bool fused_leg(size_t l) const {
        const int nx = buf.specs[l].first, ny = buf.specs[l].second;
        if (nx % 2 != 0 || leg_smem<T>(nx, ny, 2 * nit + 2, true) > kLegSmemMax ||
            leg_points(nx, ny, 2 * nit + 2) > static_cast<size_t>(2 * kLegPts * kLegThreads))
            return false;
        return static_cast<long long>(leg_grid(l).x) * batch <= leg_max_ctas<T>();
    }
    FineLeg<T> leg(size_t l, const T* uin, T* uout) const {
        double pr[5];
        params_at(l, pr);
        const MemWeights w = mem_weights(pr);
        FineLeg<T> g{};
        g.A = buf.A[l];
        g.B = buf.B[l];
        g.Uin = uin;
        g.Uout = uout;
        g.nx = buf.specs[l].first;
        g.ny = buf.specs[l].second;
        g.w00 = T(w.w00);
        g.w01 = T(w.w01);
        g.w10 = T(w.w10);
        g.rw = reg_weights(pr, 1);
        g.nB = buf.B[l + 1];
        g.nU = buf.U[l + 1];
        g.cnx = buf.specs[l + 1].first;
        g.cny = buf.specs[l + 1].second;
        g.nit = nit;
        return g;
    }
    dim3 leg_grid(size_t l) const {
        const int nx = buf.specs[l].first, ny = buf.specs[l].second;
        return dim3(static_cast<unsigned>(((nx + kTileX - 1) / kTileX) * ((ny + kTileY - 1) / kTileY)),
                    static_cast<unsigned>(batch));
    }
    void cycle(size_t start) {
        const size_t last = buf.specs.size() - 1;
        const size_t fused = std::max(start, coarse_first());
        if (buf.specs.size() <= static_cast<size_t>(kMaxLevels) && fused < last) {
            allow_big_smem<T>();
            // down: relax, residual, restriction (a fused leg leaves the relaxed solution in R[l]);
            // up: prolongation, relax (a fused leg reads R[l] and writes U[l])
            for (size_t l = start; l < fused; ++l) {
                const int nx = buf.specs[l].first, ny = buf.specs[l].second;
                if (fused_leg(l)) {
                    (csg::note_launch(), csg::launch_pdl(k_vcycle_down<T>, leg_grid(l), kLegThreads,
                                                         leg_smem<T>(nx, ny, 2 * nit + 2, true), s,
                                                         leg(l, buf.U[l], buf.R[l])));
                    continue;
                }
                relax(l);
                double pr[5];
                params_at(l, pr);
                (csg::note_launch(), csg::launch_pdl(k_membrane_apply<T>, grid_for(nx * ny, batch), kThreads, 0, s,
                                                     buf.A[l], buf.U[l], buf.B[l], buf.R[l], nx, ny, reg_weights(pr, 1)));
                resize(buf.R[l], l, buf.B[l + 1], l + 1, 2, false);
                const size_t P1 = static_cast<size_t>(buf.specs[l + 1].first) * buf.specs[l + 1].second;
                cudaMemsetAsync(buf.U[l + 1], 0, 2 * P1 * batch * sizeof(T), s);
            }
            coarse_cycle(fused);
            for (size_t l = fused; l-- > start;) {
                const int nx = buf.specs[l].first, ny = buf.specs[l].second;
                if (fused_leg(l)) {
                    (csg::note_launch(), csg::launch_pdl(k_vcycle_up<T>, leg_grid(l), kLegThreads,
                                                         leg_smem<T>(nx, ny, 2 * nit, false), s,
                                                         leg(l, buf.R[l], buf.U[l])));
                    continue;
                }
                resize(buf.U[l + 1], l + 1, buf.U[l], l, 2, true);
                relax(l);
            }
            return;
        }
        for (size_t l = start; l < last; ++l) {
            relax(l);
            const int nx = buf.specs[l].first, ny = buf.specs[l].second;
            double pr[5];
            params_at(l, pr);
            (csg::note_launch(), csg::launch_pdl(k_membrane_apply<T>, grid_for(nx * ny, batch), kThreads, 0, s, buf.A[l], buf.U[l], buf.B[l], buf.R[l], nx,
                                                                               ny, reg_weights(pr, 1)));
            resize(buf.R[l], l, buf.B[l + 1], l + 1, 2, false);
            const size_t P1 = static_cast<size_t>(buf.specs[l + 1].first) * buf.specs[l + 1].second;
            cudaMemsetAsync(buf.U[l + 1], 0, 2 * P1 * batch * sizeof(T), s);
        }
        relax(last);
        for (size_t l = last; l-- > start;) {
            resize(buf.U[l + 1], l + 1, buf.U[l], l, 2, true);
            relax(l);
        }
    }
    // Solves into buf.U[0]; U[0] must already hold the initial guess (or
    // zeros when `coarse_init`).  hess / rhs are level-0 A / B.
    // A[l] = resize(A[l - 1]) for every level: separate launches down to
    // kChainPoints points per grid, then the rest in one k_resize_chain launch.
    void restrict_hessians() {
        const size_t L = buf.specs.size();
        size_t l = 1;
        for (; l < L && static_cast<long long>(buf.specs[l].first) * buf.specs[l].second > kChainPoints; ++l)
            resize(buf.A[l - 1], l - 1, buf.A[l], l, 3, false);
        if (l >= L) return;
        if (L > static_cast<size_t>(kMaxLevels)) {
            for (; l < L; ++l) resize(buf.A[l - 1], l - 1, buf.A[l], l, 3, false);
            return;
        }
        ResizeChain<T> c{};
        for (size_t k = 0; k < L; ++k) {
            c.field[k] = buf.A[k];
            c.nx[k] = buf.specs[k].first;
            c.ny[k] = buf.specs[k].second;
        }
        c.first = static_cast<int>(l);
        c.last = static_cast<int>(L - 1);
        c.channels = 3;
        for (int k = c.first, off = 0; k <= c.last; ++k) {
            c.off[k] = off;
            off += c.channels * c.nx[k] * c.ny[k];
        }
        allow_big_smem<T>();
        (csg::note_launch(), csg::launch_pdl(k_resize_chain<T>, batch, kCoarseThreads, resize_chain_smem(c), s, c));
    }
    void run(bool coarse_init) {
        const size_t L = buf.specs.size();
        restrict_hessians();
        if (!coarse_init) {
            // every V-cycle writes each coarser level's right-hand side and zeroes its
            // solution before reading them, so the warm start needs no clearing
            for (int c = 0; c < cycles; ++c) cycle(0);
            return;
        }
        for (size_t l = 1; l < L; ++l) resize(l == 1 ? buf.B[0] : buf.B0[l - 1], l - 1, buf.B0[l], l, 2, false);
        for (size_t l = 1; l < L; ++l) {
            const size_t P = static_cast<size_t>(buf.specs[l].first) * buf.specs[l].second;
            cudaMemsetAsync(buf.B[l], 0, 2 * P * batch * sizeof(T), s);
            cudaMemsetAsync(buf.U[l], 0, 2 * P * batch * sizeof(T), s);
        }
        const size_t last = L - 1;
        const size_t Pl = static_cast<size_t>(buf.specs[last].first) * buf.specs[last].second;
        (csg::note_launch(), csg::launch_pdl(k_point_solve<T>, grid_for(static_cast<int>(Pl), batch), kThreads, 0, s, 
            buf.A[last], last == 0 ? buf.B[0] : buf.B0[last], buf.U[last], static_cast<int>(Pl), T(base[4])));
        relax(last);
        for (size_t l = last; l-- > 0;) {
            resize(buf.U[l + 1], l + 1, buf.U[l], l, 2, false);
            if (l > 0) {
                const size_t P = static_cast<size_t>(buf.specs[l].first) * buf.specs[l].second;
                cudaMemcpyAsync(buf.B[l], buf.B0[l], 2 * P * batch * sizeof(T), cudaMemcpyDeviceToDevice, s);
            }
            for (int c = 0; c < cycles; ++c) cycle(l);
        }
    }
};

// Workspace of one dartel_step for a batch.
template <typename T>
struct StepBuffers {
    T *map[2], *jac[2], *smap[2], *sjac[2], *rmap[2], *rjac[2];
    T *rhs_f[2], *hess_f[2], *rhs_r[2], *hess_r[2];
    T *rhs, *hess, *objf, *objr, *preg, *pnorm;
    FmgBuffers<T> fmg;
    int nblocks;
    bool carve(Arena& ar, int batch, int nx, int ny) {
        const size_t P = static_cast<size_t>(nx) * ny * batch;
        for (int i = 0; i < 2; ++i) {
            map[i] = ar.take<T>(2 * P);
            jac[i] = ar.take<T>(4 * P);
            smap[i] = ar.take<T>(2 * P);
            sjac[i] = ar.take<T>(4 * P);
            rmap[i] = ar.take<T>(2 * P);
            rjac[i] = ar.take<T>(4 * P);
            rhs_f[i] = ar.take<T>(2 * P);
            hess_f[i] = ar.take<T>(3 * P);
            rhs_r[i] = ar.take<T>(2 * P);
            hess_r[i] = ar.take<T>(3 * P);
        }
        nblocks = (nx * ny + kThreads - 1) / kThreads;
        objf = ar.take<T>(static_cast<size_t>(nblocks) * batch);
        objr = ar.take<T>(static_cast<size_t>(nblocks) * batch);
        preg = ar.take<T>(static_cast<size_t>(nblocks) * batch);
        pnorm = ar.take<T>(static_cast<size_t>(nblocks) * batch);
        // rhs / hess of the solve live in the multigrid's level-0 slots
        if (!fmg.carve(ar, batch, nx, ny)) return false;
        rhs = ar.take<T>(2 * P);
        hess = ar.take<T>(3 * P);
        return ar.ok;
    }
};

// squaring_update (dartel_grid.py:778-914) with the reference's two-slot
// bookkeeping: slot `other` receives each step's b increment and, when the
// map is composed, the composed map; slot 0 after the loop is the
// "scratch" dartel_step hands to the multigrid as its initial guess.
// Returns the index of the current slot; b / a end in rb[cur_ba] / ha[cur_ba].
template <typename T>
struct Squaring {
    int cur_map, cur_ba;
};

template <typename T>
Squaring<T> run_squaring(T* rb[2], T* ha[2], T* maps[2], T* jacs[2], int k, bool save, int batch, int nx, int ny,
                         cudaStream_t s) {
    const dim3 g = grid_for(nx * ny, batch);
    int cur = 0, other = 1, ba = 0;
    for (int step = 0; step < k; ++step) {
        if (save || step < k - 1) {
            (csg::note_launch(), csg::launch_pdl(k_squaring_compose<T>, g, kThreads, 0, s, rb[ba], ha[ba], maps[cur],
                                                 jacs[cur], rb[1 - ba], ha[1 - ba], maps[other], jacs[other], nx, ny));
            std::swap(cur, other);
        } else {
            (csg::note_launch(), csg::launch_pdl(k_squaring<T>, g, kThreads, 0, s, rb[ba], ha[ba], maps[cur], jacs[cur],
                                                 rb[1 - ba], ha[1 - ba], maps[other], nx, ny));
        }
        ba = 1 - ba;
    }
    if (save && cur != 0) {
        const size_t P = static_cast<size_t>(nx) * ny * batch;
        cudaMemcpyAsync(maps[0], maps[cur], 2 * P * sizeof(T), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(jacs[0], jacs[cur], 4 * P * sizeof(T), cudaMemcpyDeviceToDevice, s);
    }
    return {cur, ba};
}

template <typename T>
int dartel_step_impl(StepBuffers<T>& W, const T* source, const T* target, T* velocity, T* metrics, int metric_stride,
                     int batch, int nx, int ny, int k, const double* params, double lmreg, int cycles, int nit,
                     int code, int assume_initial_nonzero, cudaStream_t s) {
    const dim3 g = grid_for(nx * ny, batch);
    const double scale = 1.0 / static_cast<double>(1LL << k);
    const size_t P = static_cast<size_t>(nx) * ny * batch;
    // expdef(v, k) with Jacobian
    (csg::note_launch(), csg::launch_pdl(k_smalldef<T>, g, kThreads, 0, s, velocity, W.map[0], W.jac[0], nx, ny, T(scale), T(scale * 0.5)));
    int cur = 0;
    for (int i = 0; i < k; ++i) {
        (csg::note_launch(), csg::launch_pdl(k_compose<T>, g, kThreads, 0, s, W.map[cur], W.jac[cur], W.map[cur], W.jac[cur], W.map[1 - cur],
                                            W.jac[1 - cur], nx, ny));
        cur = 1 - cur;
    }
    // forward objective with jac_div_smalldef(J, v, s)
    (csg::note_launch(), csg::launch_pdl(k_objfun<T, true>, g, kThreads, 0, s, source, target, W.map[cur], W.jac[cur], velocity, nullptr, W.rhs_f[0],
                                             W.hess_f[0], W.objf, nx, ny, T(scale * 0.5)));
    // squaring of the forward terms from smalldef_jac(v, -s)
    (csg::note_launch(), csg::launch_pdl(k_smalldef<T>, g, kThreads, 0, s, velocity, W.smap[0], W.sjac[0], nx, ny, T(-scale), T(-scale * 0.5)));
    Squaring<T> fw = run_squaring<T>(W.rhs_f, W.hess_f, W.smap, W.sjac, k, code == 1, batch, nx, ny, s);
    T* initial = W.smap[0];
    T* rr = nullptr;
    T* hr = nullptr;
    if (code == 1) {
        (csg::note_launch(), csg::launch_pdl(k_objfun<T, true>, g, kThreads, 0, s, target, source, W.smap[fw.cur_map], W.sjac[fw.cur_map], velocity,
                                                 nullptr, W.rhs_r[0], W.hess_r[0], W.objr, nx, ny, T(-scale * 0.5)));
        (csg::note_launch(), csg::launch_pdl(k_smalldef<T>, g, kThreads, 0, s, velocity, W.rmap[0], W.rjac[0], nx, ny, T(scale), T(scale * 0.5)));
        Squaring<T> rv = run_squaring<T>(W.rhs_r, W.hess_r, W.rmap, W.rjac, k, false, batch, nx, ny, s);
        initial = W.rmap[0];
        rr = W.rhs_r[rv.cur_ba];
        hr = W.hess_r[rv.cur_ba];
    }
    const RegWeights rw = reg_weights(params, 1);
    T* rhs = W.rhs;
    (csg::note_launch(), csg::launch_pdl(k_combine<T>, g, kThreads, 0, s, W.rhs_f[fw.cur_ba], rr, W.hess_f[fw.cur_ba], hr, velocity, rhs, W.hess, W.preg,
                                        W.pnorm, nx, ny, T(scale), rw));
    (csg::note_launch(), csg::launch_pdl(k_metrics<T>, batch, 32, 0, s, W.objf, code == 1 ? W.objr : nullptr, W.preg, W.pnorm, W.nblocks, metrics,
                                      metric_stride));
    // multigrid solve of (H + L) u = rhs from the scratch initial guess
    double solver[5] = {params[0], params[1], params[2], params[3], params[4] + lmreg};
    Fmg<T> fmg{W.fmg, batch, {solver[0], solver[1], solver[2], solver[3], solver[4]}, cycles, nit, s, nx, ny};
    W.fmg.A[0] = W.hess;
    W.fmg.B[0] = rhs;
    W.fmg.U[0] = initial;
    bool coarse_init = false;
    if (!assume_initial_nonzero) {
        int flag = 0;
        CSG_CUDA_CHECK(cudaMemsetAsync(W.fmg.flag, 0, sizeof(int), s));
        (csg::note_launch(), csg::launch_pdl(k_any_nonzero<T>, static_cast<unsigned>((2 * P + kThreads - 1) / kThreads), kThreads, 0, s, initial, 2 * P,
                                                                                                     W.fmg.flag));
        CSG_CUDA_CHECK(cudaMemcpyAsync(&flag, W.fmg.flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        CSG_CUDA_CHECK(cudaStreamSynchronize(s));
        coarse_init = flag == 0;
        if (coarse_init) CSG_CUDA_CHECK(cudaMemsetAsync(initial, 0, 2 * P * sizeof(T), s));
    }
    fmg.run(coarse_init);
    (csg::note_launch(), csg::launch_pdl(k_sub<T>, static_cast<unsigned>((2 * P + kThreads - 1) / kThreads), kThreads, 0, s, velocity, initial, 2 * P));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

size_t dtype_size(int dtype) { return dtype == CSG_DTYPE_F64 ? 8 : 4; }

bool check_dtype(int dtype) { return dtype == CSG_DTYPE_F32 || dtype == CSG_DTYPE_F64; }

template <typename T>
size_t step_bytes(int batch, int nx, int ny) {
    Arena ar{nullptr, static_cast<size_t>(-1) / 2};
    StepBuffers<T> W;
    W.carve(ar, batch, nx, ny);
    return ar.used + 256;
}

template <typename T>
size_t expdef_bytes(int batch, int nx, int ny) {
    return 2 * (2 + 4) * static_cast<size_t>(nx) * ny * batch * sizeof(T) + 1024;
}

template <typename T>
int solve_typed(const void* source, const void* target, void* velocity, void* metrics, int batch, int nx,
                       int ny, int loop, const double* params, int its, double lmreg, int cycles, int nit, int code,
                       int assume, void* scratch, size_t bytes, cudaStream_t s) {
    Arena ar{static_cast<char*>(scratch), bytes};
    StepBuffers<T> W;
    if (!W.carve(ar, batch, nx, ny)) return csg::fail(CSG_ERR_ARG, "dartel: scratch of %zu bytes is too small", bytes);
    const int per = loop * its;
    for (int index = 0; index < loop; ++index)
        for (int it = 0; it < its; ++it) {
            int rc = dartel_step_impl<T>(W, static_cast<const T*>(source), static_cast<const T*>(target),
                                         static_cast<T*>(velocity), static_cast<T*>(metrics) + 3 * (index * its + it),
                                         3 * per, batch, nx, ny, index, params + 5 * index, lmreg, cycles, nit, code,
                                         assume, s);
            if (rc) return rc;
        }
    return CSG_OK;
}

int check_grid(int dtype, int batch, int nx, int ny) {
    if (!check_dtype(dtype)) return csg::fail(CSG_ERR_ARG, "dartel: dtype must be CSG_DTYPE_F32 or CSG_DTYPE_F64");
    if (batch < 1 || nx < 1 || ny < 1) return csg::fail(CSG_ERR_ARG, "dartel: empty grid (%d x %d x %d)", batch, ny, nx);
    if (static_cast<long long>(nx) * ny > (1LL << 30)) return csg::fail(CSG_ERR_ARG, "dartel: grid too large");
    return CSG_OK;
}

// ------------------------------------------------ data-term adjoint
//
// E_b(v) = 1/2 sum_x (S_b(phi_k(x)) - T_b(x))^2 with phi_0 = id + v / 2^k and
// phi_{i+1} = phi_i o phi_i (the forward maps of expdef).  The adjoint runs
// the same bilinear stencils backwards: the sample step gives
// abar = r grad S(phi_k); each composition step C = F(A) with A = phi_i(x)
// and F = phi_i splits abar into the position part J_F(A)^T abar (added at
// x) and the value part (scattered to the four corner nodes with the
// bilinear weights, atomically).  The period unwrap of the corner values is
// a piecewise constant shift, so its derivative is the identity.

// Residual of one sample step, its block objective partial and (when abar is
// non-null) abar = r (dS/dX, dS/dY).
template <typename T>
__global__ void k_data_sample(const T* __restrict__ source, const T* __restrict__ target, const T* __restrict__ map,
                              T* __restrict__ abar, T* __restrict__ partial, int nx, int ny) {
    csg::pdl_begin();
    Pt p;
    const bool ok = point(nx, ny, p);
    T contrib = T(0);
    if (ok) {
        const int P = nx * ny;
        const size_t o1 = static_cast<size_t>(p.b) * P;
        const T* src = source + o1;
        const T* M = map + 2 * o1;
        const Stencil<T> st(M[p.i] - T(1), M[P + p.i] - T(1), nx, ny);
        const T k22 = src[st.i22], k12 = src[st.i12], k21 = src[st.i21], k11 = src[st.i11];
        const T sampled = (k22 * st.dx2 + k12 * st.dx1) * st.dy2 + (k21 * st.dx2 + k11 * st.dx1) * st.dy1;
        const T r = sampled - target[o1 + p.i];
        if (abar) {
            const T ddx = (k11 - k21) * st.dy1 + (k12 - k22) * st.dy2;
            const T ddy = (k11 * st.dx1 + k21 * st.dx2) - (k12 * st.dx1 + k22 * st.dx2);
            abar[2 * o1 + p.i] = r * ddx;
            abar[2 * o1 + P + p.i] = r * ddy;
        }
        contrib = r * r;
    }
    block_sum(contrib, partial);
}

// objective[b] = 1/2 sum of the block partials of batch b, in block order.
template <typename T>
__global__ void k_data_objective(const T* __restrict__ partial, int nblocks, int batch, T* __restrict__ objective) {
    csg::pdl_begin();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    T total = T(0);
    for (int i = 0; i < nblocks; ++i) total = total + partial[static_cast<size_t>(b) * nblocks + i];
    objective[b] = total * T(0.5);
}

// pbar += adjoint of C = phi_i o phi_i at every x (pbar zeroed by the caller).
template <typename T>
__global__ void k_data_compose_adjoint(const T* __restrict__ f, const T* __restrict__ abar, T* __restrict__ pbar,
                                       int nx, int ny) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const size_t o2 = static_cast<size_t>(p.b) * 2 * P;
    const T* F = f + o2;
    const Stencil<T> st(F[p.i] - T(1), F[P + p.i] - T(1), nx, ny);
    T* out = pbar + o2;
    T pos_x = T(0), pos_y = T(0);
#pragma unroll
    for (int ch = 0; ch < 2; ++ch) {
        const T* fc = F + ch * P;
        const T period = static_cast<T>(ch == 0 ? nx : ny);
        const T c22 = fc[st.i22] - T(1);
        const T c12 = unwrap(fc[st.i12] - T(1), c22, period);
        const T c21 = unwrap(fc[st.i21] - T(1), c22, period);
        const T c11 = unwrap(fc[st.i11] - T(1), c22, period);
        const T a = abar[o2 + ch * P + p.i];
        pos_x = pos_x + a * ((c12 - c22) * st.dy2 + (c11 - c21) * st.dy1);
        pos_y = pos_y + a * ((c21 * st.dx2 + c11 * st.dx1) - (c22 * st.dx2 + c12 * st.dx1));
        T* oc = out + ch * P;
        atomicAdd(oc + st.i22, a * (st.dx2 * st.dy2));
        atomicAdd(oc + st.i12, a * (st.dx1 * st.dy2));
        atomicAdd(oc + st.i21, a * (st.dx2 * st.dy1));
        atomicAdd(oc + st.i11, a * (st.dx1 * st.dy1));
    }
    atomicAdd(out + p.i, pos_x);
    atomicAdd(out + P + p.i, pos_y);
}

// grad = scale_b * s * abar (phi_0 = id + s v).
template <typename T>
__global__ void k_data_velocity_grad(const T* __restrict__ abar, const T* __restrict__ grad_scale, T s,
                                     T* __restrict__ grad, int nx, int ny) {
    csg::pdl_begin();
    Pt p;
    if (!point(nx, ny, p)) return;
    const int P = nx * ny;
    const size_t o2 = static_cast<size_t>(p.b) * 2 * P;
    const T g = grad_scale ? grad_scale[p.b] * s : s;
    grad[o2 + p.i] = abar[o2 + p.i] * g;
    grad[o2 + P + p.i] = abar[o2 + P + p.i] * g;
}

inline int data_checkpoints(int k, int every) { return k == 0 ? 1 : (k - 1) / every + 1; }

inline size_t align_up(size_t bytes) { return (bytes + 255) & ~static_cast<size_t>(255); }

template <typename T>
size_t data_scratch(int batch, int nx, int ny, int k, int every) {
    const size_t field = align_up(sizeof(T) * 2ULL * batch * nx * ny);
    const size_t nblocks = (static_cast<size_t>(nx) * ny + kThreads - 1) / kThreads;
    // forward ping-pong 2, backward segment `every`, abar + pbar, block partials
    return field * (2 + static_cast<size_t>(every) + 2) + align_up(sizeof(T) * nblocks * batch) + 256;
}

template <typename T>
struct DataScratch {
    T* work[2];
    T* seg;  // `every` maps
    T* abar;
    T* pbar;
    T* partial;
    size_t field_elems;
};

template <typename T>
DataScratch<T> carve_data(void* scratch, int batch, int nx, int ny, int every) {
    DataScratch<T> d{};
    const size_t field = align_up(sizeof(T) * 2ULL * batch * nx * ny);
    char* base = static_cast<char*>(scratch);
    d.work[0] = reinterpret_cast<T*>(base);
    d.work[1] = reinterpret_cast<T*>(base + field);
    d.seg = reinterpret_cast<T*>(base + 2 * field);
    d.abar = reinterpret_cast<T*>(base + (2 + static_cast<size_t>(every)) * field);
    d.pbar = reinterpret_cast<T*>(base + (3 + static_cast<size_t>(every)) * field);
    d.partial = reinterpret_cast<T*>(base + (4 + static_cast<size_t>(every)) * field);
    d.field_elems = field / sizeof(T);
    return d;
}

template <typename T>
int data_forward_typed(int batch, int nx, int ny, const T* v, const T* source, const T* target, int k, int every,
                       T* checkpoints, T* objective, void* scratch, size_t bytes, cudaStream_t s) {
    if (bytes < data_scratch<T>(batch, nx, ny, k, every)) return csg::fail(CSG_ERR_ARG, "data term: scratch too small");
    DataScratch<T> d = carve_data<T>(scratch, batch, nx, ny, every);
    const size_t field = 2ULL * batch * nx * ny;
    const dim3 g = grid_for(nx * ny, batch);
    const T step = static_cast<T>(std::ldexp(1.0, -k));
    (csg::note_launch(), csg::launch_pdl(k_smalldef<T>, g, kThreads, 0, s, v, checkpoints, nullptr, nx, ny, step, T(0)));
    const T* cur = checkpoints;
    for (int i = 1; i <= k; ++i) {
        T* dst = (i % every == 0 && i < k) ? checkpoints + field * (i / every) : d.work[i % 2];
        (csg::note_launch(), csg::launch_pdl(k_compose<T>, g, kThreads, 0, s, cur, nullptr, cur, nullptr, dst, nullptr, nx, ny));
        cur = dst;
    }
    (csg::note_launch(), csg::launch_pdl(k_data_sample<T>, g, kThreads, 0, s, source, target, cur, nullptr, d.partial, nx, ny));
    (csg::note_launch(), csg::launch_pdl(k_data_objective<T>, (batch + 127) / 128, 128, 0, s, d.partial, static_cast<int>(g.x), batch,
                                                                               objective));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

template <typename T>
int data_backward_typed(int batch, int nx, int ny, const T* source, const T* target, int k, int every,
                        const T* checkpoints, const T* grad_scale, T* grad, void* scratch, size_t bytes,
                        cudaStream_t s) {
    if (bytes < data_scratch<T>(batch, nx, ny, k, every)) return csg::fail(CSG_ERR_ARG, "data term: scratch too small");
    DataScratch<T> d = carve_data<T>(scratch, batch, nx, ny, every);
    const size_t field = 2ULL * batch * nx * ny;
    const dim3 g = grid_for(nx * ny, batch);
    const int n_ckpt = data_checkpoints(k, every);
    T* abar = d.abar;
    T* pbar = d.pbar;
    std::vector<const T*> maps(static_cast<size_t>(every) + 1);
    for (int j = n_ckpt - 1; j >= 0; --j) {
        const int first = j * every;
        const int last = (j == n_ckpt - 1) ? k : (j + 1) * every - 1;  // maps this segment needs
        maps[0] = checkpoints + field * j;
        for (int i = first + 1; i <= last; ++i) {
            T* dst = d.seg + d.field_elems * static_cast<size_t>(i - first - 1);
            (csg::note_launch(), csg::launch_pdl(k_compose<T>, g, kThreads, 0, s, maps[i - first - 1], nullptr, maps[i - first - 1],
                                                                   nullptr, dst, nullptr, nx, ny));
            maps[i - first] = dst;
        }
        if (j == n_ckpt - 1)
            (csg::note_launch(), csg::launch_pdl(k_data_sample<T>, g, kThreads, 0, s, source, target, maps[k - first], abar,
                                                                       d.partial, nx, ny));
        const int top = (j == n_ckpt - 1) ? k - 1 : last;
        for (int i = top; i >= first; --i) {
            CSG_CUDA_CHECK(cudaMemsetAsync(pbar, 0, sizeof(T) * field, s));
            (csg::note_launch(), csg::launch_pdl(k_data_compose_adjoint<T>, g, kThreads, 0, s, maps[i - first], abar, pbar, nx, ny));
            T* t = abar;
            abar = pbar;
            pbar = t;
        }
    }
    const T step = static_cast<T>(std::ldexp(1.0, -k));
    (csg::note_launch(), csg::launch_pdl(k_data_velocity_grad<T>, g, kThreads, 0, s, abar, grad_scale, step, grad, nx, ny));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int check_levels(int nx, int ny) {
    for (const auto& spec : grid_levels(nx, ny))
        if (!relax_supported(spec.first))
            return csg::fail(CSG_ERR_UNSUPPORTED,
                             "dartel: red-black relaxation needs an even x size on every multigrid level "
                             "(level %d x %d)", spec.second, spec.first);
    return CSG_OK;
}

}  // namespace

extern "C" {

size_t csg_dartel_scratch_bytes(int dtype, int batch, int nx, int ny) {
    if (!check_dtype(dtype) || batch < 1 || nx < 1 || ny < 1) return 0;
    return dtype == CSG_DTYPE_F64 ? step_bytes<double>(batch, nx, ny) : step_bytes<float>(batch, nx, ny);
}

int csg_dartel_solve(int dtype, int batch, int nx, int ny, const void* source_maps, const void* target_maps,
                     void* velocity, void* metrics, int loop, const double* params, int its, double lmreg, int cycles,
                     int nit, int code, int assume_initial_nonzero, void* scratch, size_t scratch_bytes,
                     csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!source_maps || !target_maps || !velocity || !metrics || !params || !scratch)
        return csg::fail(CSG_ERR_ARG, "dartel solve: null pointer");
    if (loop < 1 || its < 0 || cycles < 0 || nit < 0 || (code != 0 && code != 1) || loop > 30)
        return csg::fail(CSG_ERR_ARG, "dartel solve: bad loop/its/cycles/nit/code");
    rc = check_levels(nx, ny);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F64)
        return solve_typed<double>(source_maps, target_maps, velocity, metrics, batch, nx, ny, loop, params, its, lmreg,
                                   cycles, nit, code, assume_initial_nonzero, scratch, scratch_bytes, s);
    return solve_typed<float>(source_maps, target_maps, velocity, metrics, batch, nx, ny, loop, params, its, lmreg,
                              cycles, nit, code, assume_initial_nonzero, scratch, scratch_bytes, s);
}

int csg_dartel_step(int dtype, int batch, int nx, int ny, const void* source, const void* target, void* velocity,
                    void* metrics, int k, const double* params, double lmreg, int cycles, int nit, int code,
                    int assume_initial_nonzero, void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!source || !target || !velocity || !metrics || !params || !scratch)
        return csg::fail(CSG_ERR_ARG, "dartel step: null pointer");
    if (k < 0 || k > 30 || cycles < 0 || nit < 0 || (code != 0 && code != 1))
        return csg::fail(CSG_ERR_ARG, "dartel step: bad k/cycles/nit/code");
    rc = check_levels(nx, ny);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F64) {
        Arena ar{static_cast<char*>(scratch), scratch_bytes};
        StepBuffers<double> W;
        if (!W.carve(ar, batch, nx, ny)) return csg::fail(CSG_ERR_ARG, "dartel step: scratch too small");
        return dartel_step_impl<double>(W, static_cast<const double*>(source), static_cast<const double*>(target),
                                        static_cast<double*>(velocity), static_cast<double*>(metrics), 3, batch, nx, ny,
                                        k, params, lmreg, cycles, nit, code, assume_initial_nonzero, s);
    }
    Arena ar{static_cast<char*>(scratch), scratch_bytes};
    StepBuffers<float> W;
    if (!W.carve(ar, batch, nx, ny)) return csg::fail(CSG_ERR_ARG, "dartel step: scratch too small");
    return dartel_step_impl<float>(W, static_cast<const float*>(source), static_cast<const float*>(target),
                                   static_cast<float*>(velocity), static_cast<float*>(metrics), 3, batch, nx, ny, k,
                                   params, lmreg, cycles, nit, code, assume_initial_nonzero, s);
}

}  // extern "C"

// ------------------------------------------------------- single operators

namespace {

template <typename T>
int smalldef_typed(int batch, int nx, int ny, const void* v, double scale, void* map, void* jac, cudaStream_t s) {
    (csg::note_launch(), csg::launch_pdl(k_smalldef<T>, grid_for(nx * ny, batch), kThreads, 0, s, static_cast<const T*>(v), static_cast<T*>(map),
                                                                 static_cast<T*>(jac), nx, ny, T(scale), T(scale * 0.5)));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

template <typename T>
int squaring_typed(int batch, int nx, int ny, const void* rhs, const void* hess, const void* map, const void* jac,
                   int k, int save, void* b_out, void* a_out, void* map_out, void* jac_out, void* scratch_out,
                   void* work, size_t bytes, cudaStream_t s) {
    const size_t P = static_cast<size_t>(nx) * ny * batch;
    Arena ar{static_cast<char*>(work), bytes};
    T *rb[2], *ha[2], *maps[2], *jacs[2];
    for (int i = 0; i < 2; ++i) {
        rb[i] = ar.take<T>(2 * P);
        ha[i] = ar.take<T>(3 * P);
        maps[i] = ar.take<T>(2 * P);
        jacs[i] = ar.take<T>(4 * P);
    }
    if (!ar.ok) return csg::fail(CSG_ERR_ARG, "squaring: scratch too small");
    CSG_CUDA_CHECK(cudaMemcpyAsync(rb[0], rhs, 2 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(ha[0], hess, 3 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(maps[0], map, 2 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(jacs[0], jac, 4 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    Squaring<T> r = run_squaring<T>(rb, ha, maps, jacs, k, save != 0, batch, nx, ny, s);
    CSG_CUDA_CHECK(cudaMemcpyAsync(b_out, rb[r.cur_ba], 2 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    CSG_CUDA_CHECK(cudaMemcpyAsync(a_out, ha[r.cur_ba], 3 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    if (map_out) CSG_CUDA_CHECK(cudaMemcpyAsync(map_out, maps[r.cur_map], 2 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    if (jac_out) CSG_CUDA_CHECK(cudaMemcpyAsync(jac_out, jacs[r.cur_map], 4 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    if (scratch_out) CSG_CUDA_CHECK(cudaMemcpyAsync(scratch_out, maps[0], 2 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

template <typename T>
int expdef_typed(int batch, int nx, int ny, const void* v, int k, void* map_out, void* jac_out, void* work, size_t bytes,
                 cudaStream_t s) {
    const size_t P = static_cast<size_t>(nx) * ny * batch;
    Arena ar{static_cast<char*>(work), bytes};
    T* maps[2] = {ar.take<T>(2 * P), ar.take<T>(2 * P)};
    T* jacs[2] = {ar.take<T>(4 * P), ar.take<T>(4 * P)};
    if (!ar.ok) return csg::fail(CSG_ERR_ARG, "expdef: scratch too small");
    const double scale = 1.0 / static_cast<double>(1LL << k);
    const dim3 g = grid_for(nx * ny, batch);
    const bool with_jac = jac_out != nullptr;
    (csg::note_launch(), csg::launch_pdl(k_smalldef<T>, g, kThreads, 0, s, static_cast<const T*>(v), maps[0], with_jac ? jacs[0] : nullptr, nx, ny,
                                         T(scale), T(scale * 0.5)));
    int cur = 0;
    for (int i = 0; i < k; ++i) {
        (csg::note_launch(), csg::launch_pdl(k_compose<T>, g, kThreads, 0, s, maps[cur], with_jac ? jacs[cur] : nullptr, maps[cur],
                                            with_jac ? jacs[cur] : nullptr, maps[1 - cur],
                                            with_jac ? jacs[1 - cur] : nullptr, nx, ny));
        cur = 1 - cur;
    }
    CSG_CUDA_CHECK(cudaMemcpyAsync(map_out, maps[cur], 2 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    if (with_jac) CSG_CUDA_CHECK(cudaMemcpyAsync(jac_out, jacs[cur], 4 * P * sizeof(T), cudaMemcpyDeviceToDevice, s));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

template <typename T>
int fmg_typed(int batch, int nx, int ny, const void* hess, const void* rhs, const double* params, int cycles, int nit,
              void* u, int has_initial, int assume_nonzero, void* work, size_t bytes, cudaStream_t s) {
    const size_t P = static_cast<size_t>(nx) * ny * batch;
    Arena ar{static_cast<char*>(work), bytes};
    FmgBuffers<T> buf;
    if (!buf.carve(ar, batch, nx, ny)) return csg::fail(CSG_ERR_ARG, "fmg: scratch too small");
    buf.A[0] = const_cast<T*>(static_cast<const T*>(hess));
    buf.B[0] = const_cast<T*>(static_cast<const T*>(rhs));
    buf.U[0] = static_cast<T*>(u);
    bool coarse_init = !has_initial;
    if (has_initial && !assume_nonzero) {
        int flag = 0;
        CSG_CUDA_CHECK(cudaMemsetAsync(buf.flag, 0, sizeof(int), s));
        (csg::note_launch(), csg::launch_pdl(k_any_nonzero<T>, static_cast<unsigned>((2 * P + kThreads - 1) / kThreads), kThreads, 0, s, buf.U[0], 2 * P,
                                                                                                     buf.flag));
        CSG_CUDA_CHECK(cudaMemcpyAsync(&flag, buf.flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        CSG_CUDA_CHECK(cudaStreamSynchronize(s));
        coarse_init = flag == 0;
    }
    if (coarse_init) CSG_CUDA_CHECK(cudaMemsetAsync(u, 0, 2 * P * sizeof(T), s));
    Fmg<T> fmg{buf, batch, {params[0], params[1], params[2], params[3], params[4]}, cycles, nit, s, nx, ny};
    fmg.run(coarse_init);
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

}  // namespace

extern "C" {

int csg_dartel_smalldef(int dtype, int batch, int nx, int ny, const void* velocity, double scale, void* map_out,
                        void* jac_out, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!velocity || (!map_out && !jac_out)) return csg::fail(CSG_ERR_ARG, "smalldef: null pointer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    return dtype == CSG_DTYPE_F64 ? smalldef_typed<double>(batch, nx, ny, velocity, scale, map_out, jac_out, s)
                                  : smalldef_typed<float>(batch, nx, ny, velocity, scale, map_out, jac_out, s);
}

int csg_dartel_compose(int dtype, int batch, int nx, int ny, const void* a, const void* ja, const void* b,
                       const void* jb, void* c_out, void* jc_out, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!a || !b || !c_out || ((ja != nullptr) != (jb != nullptr)) || ((ja != nullptr) != (jc_out != nullptr)))
        return csg::fail(CSG_ERR_ARG, "compose: null pointer or partial Jacobian set");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const dim3 g = grid_for(nx * ny, batch);
    if (dtype == CSG_DTYPE_F64)
        (csg::note_launch(), csg::launch_pdl(k_compose<double>, g, kThreads, 0, s, static_cast<const double*>(a), static_cast<const double*>(ja),
                                                 static_cast<const double*>(b), static_cast<const double*>(jb),
                                                 static_cast<double*>(c_out), static_cast<double*>(jc_out), nx, ny));
    else
        (csg::note_launch(), csg::launch_pdl(k_compose<float>, g, kThreads, 0, s, static_cast<const float*>(a), static_cast<const float*>(ja),
                                                static_cast<const float*>(b), static_cast<const float*>(jb),
                                                static_cast<float*>(c_out), static_cast<float*>(jc_out), nx, ny));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_dartel_jac_div(int dtype, int batch, int nx, int ny, const void* jac, const void* velocity, double scale,
                       void* out, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!jac || !velocity || !out) return csg::fail(CSG_ERR_ARG, "jac_div: null pointer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const dim3 g = grid_for(nx * ny, batch);
    if (dtype == CSG_DTYPE_F64)
        (csg::note_launch(), csg::launch_pdl(k_jacdiv<double>, g, kThreads, 0, s, static_cast<const double*>(jac), static_cast<const double*>(velocity),
                                                static_cast<double*>(out), nx, ny, scale * 0.5));
    else
        (csg::note_launch(), csg::launch_pdl(k_jacdiv<float>, g, kThreads, 0, s, static_cast<const float*>(jac), static_cast<const float*>(velocity),
                                               static_cast<float*>(out), nx, ny, static_cast<float>(scale * 0.5)));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_dartel_objfun(int dtype, int batch, int nx, int ny, const void* source, const void* target, const void* map,
                      const void* jac, const void* weights, void* rhs_out, void* hess_out, void* objective_out,
                      void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!source || !target || !map || !jac || !rhs_out || !hess_out || !objective_out || !scratch)
        return csg::fail(CSG_ERR_ARG, "objfun: null pointer");
    const int nblocks = (nx * ny + kThreads - 1) / kThreads;
    if (scratch_bytes < static_cast<size_t>(nblocks) * batch * dtype_size(dtype))
        return csg::fail(CSG_ERR_ARG, "objfun: scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const dim3 g = grid_for(nx * ny, batch);
    if (dtype == CSG_DTYPE_F64) {
        (csg::note_launch(), csg::launch_pdl(k_objfun<double, false>, g, kThreads, 0, s, 
            static_cast<const double*>(source), static_cast<const double*>(target), static_cast<const double*>(map),
            static_cast<const double*>(jac), nullptr, static_cast<const double*>(weights), static_cast<double*>(rhs_out),
            static_cast<double*>(hess_out), static_cast<double*>(scratch), nx, ny, 0.0));
        (csg::note_launch(), csg::launch_pdl(k_objective_out<double>, batch, 32, 0, s, static_cast<double*>(scratch), nblocks,
                                                     static_cast<double*>(objective_out)));
    } else {
        (csg::note_launch(), csg::launch_pdl(k_objfun<float, false>, g, kThreads, 0, s, 
            static_cast<const float*>(source), static_cast<const float*>(target), static_cast<const float*>(map),
            static_cast<const float*>(jac), nullptr, static_cast<const float*>(weights), static_cast<float*>(rhs_out),
            static_cast<float*>(hess_out), static_cast<float*>(scratch), nx, ny, 0.0f));
        (csg::note_launch(), csg::launch_pdl(k_objective_out<float>, batch, 32, 0, s, static_cast<float*>(scratch), nblocks,
                                                    static_cast<float*>(objective_out)));
    }
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_dartel_squaring(int dtype, int batch, int nx, int ny, const void* rhs, const void* hess, const void* map,
                        const void* jac, int k, int save_transformation, void* b_out, void* a_out, void* map_out,
                        void* jac_out, void* scratch_map_out, void* scratch, size_t scratch_bytes,
                        csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!rhs || !hess || !map || !jac || !b_out || !a_out || !scratch || k < 0 || k > 30)
        return csg::fail(CSG_ERR_ARG, "squaring: null pointer or bad k");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F64)
        return squaring_typed<double>(batch, nx, ny, rhs, hess, map, jac, k, save_transformation, b_out, a_out, map_out,
                                      jac_out, scratch_map_out, scratch, scratch_bytes, s);
    return squaring_typed<float>(batch, nx, ny, rhs, hess, map, jac, k, save_transformation, b_out, a_out, map_out,
                                 jac_out, scratch_map_out, scratch, scratch_bytes, s);
}

int csg_dartel_regularization(int dtype, int batch, int nx, int ny, const void* velocity, const double* params,
                              int rtype, void* out, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!velocity || !params || !out || rtype < 0 || rtype > 2)
        return csg::fail(CSG_ERR_ARG, "regularization: null pointer or rtype not in {0, 1, 2}");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const RegWeights rw = reg_weights(params, rtype);
    const dim3 g = grid_for(nx * ny, batch);
    if (dtype == CSG_DTYPE_F64)
        (csg::note_launch(), csg::launch_pdl(k_regularise<double>, g, kThreads, 0, s, static_cast<const double*>(velocity), static_cast<double*>(out), nx,
                                                    ny, rtype, rw));
    else
        (csg::note_launch(), csg::launch_pdl(k_regularise<float>, g, kThreads, 0, s, static_cast<const float*>(velocity), static_cast<float*>(out), nx, ny,
                                                   rtype, rw));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_dartel_membrane_apply(int dtype, int batch, int nx, int ny, const void* hess, const void* field,
                              const double* params, void* out, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!hess || !field || !params || !out) return csg::fail(CSG_ERR_ARG, "membrane apply: null pointer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const RegWeights rw = reg_weights(params, 1);
    const dim3 g = grid_for(nx * ny, batch);
    if (dtype == CSG_DTYPE_F64)
        (csg::note_launch(), csg::launch_pdl(k_membrane_apply<double>, g, kThreads, 0, s, static_cast<const double*>(hess), static_cast<const double*>(field),
                                                        nullptr, static_cast<double*>(out), nx, ny, rw));
    else
        (csg::note_launch(), csg::launch_pdl(k_membrane_apply<float>, g, kThreads, 0, s, static_cast<const float*>(hess), static_cast<const float*>(field),
                                                       nullptr, static_cast<float*>(out), nx, ny, rw));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_dartel_relax(int dtype, int batch, int nx, int ny, const void* hess, const void* rhs, const double* params,
                     int nit, void* u, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!hess || !rhs || !params || !u || nit < 0) return csg::fail(CSG_ERR_ARG, "relax: null pointer or nit < 0");
    if (!relax_supported(nx))
        return csg::fail(CSG_ERR_UNSUPPORTED, "relax: red-black relaxation on the GPU needs an even x size (got %d)", nx);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const MemWeights w = mem_weights(params);
    const dim3 g = grid_for(nx * ny, batch);
    for (int it = 0; it < 2 * nit; ++it) {
        const int colour = it % 2 == 0 ? 1 : 0;
        if (dtype == CSG_DTYPE_F64)
            (csg::note_launch(), csg::launch_pdl(k_relax<double>, g, kThreads, 0, s, static_cast<const double*>(hess), static_cast<const double*>(rhs),
                                                   static_cast<double*>(u), nx, ny, colour, w.w00, w.w01, w.w10));
        else
            (csg::note_launch(), csg::launch_pdl(k_relax<float>, g, kThreads, 0, s, static_cast<const float*>(hess), static_cast<const float*>(rhs),
                                                  static_cast<float*>(u), nx, ny, colour, static_cast<float>(w.w00),
                                                  static_cast<float>(w.w01), static_cast<float>(w.w10)));
    }
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_dartel_resize(int dtype, int fields, int src_nx, int src_ny, const void* src, int dst_nx, int dst_ny,
                      void* dst, int accumulate, csg_stream_t stream) {
    if (!check_dtype(dtype) || fields < 1 || src_nx < 1 || src_ny < 1 || dst_nx < 1 || dst_ny < 1 || !src || !dst)
        return csg::fail(CSG_ERR_ARG, "resize: bad arguments");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const dim3 g = grid_for(dst_nx * dst_ny, fields);
    if (dtype == CSG_DTYPE_F64)
        (csg::note_launch(), csg::launch_pdl(k_resize<double>, g, kThreads, 0, s, static_cast<const double*>(src), static_cast<double*>(dst), src_nx,
                                                src_ny, dst_nx, dst_ny, accumulate));
    else
        (csg::note_launch(), csg::launch_pdl(k_resize<float>, g, kThreads, 0, s, static_cast<const float*>(src), static_cast<float*>(dst), src_nx, src_ny,
                                               dst_nx, dst_ny, accumulate));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_dartel_fmg(int dtype, int batch, int nx, int ny, const void* hess, const void* rhs, const double* params,
                   int cycles, int nit, void* u, int has_initial, int assume_initial_nonzero, void* scratch,
                   size_t scratch_bytes, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!hess || !rhs || !params || !u || !scratch || cycles < 0 || nit < 0)
        return csg::fail(CSG_ERR_ARG, "fmg: null pointer or negative cycles / nit");
    rc = check_levels(nx, ny);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F64)
        return fmg_typed<double>(batch, nx, ny, hess, rhs, params, cycles, nit, u, has_initial, assume_initial_nonzero,
                                 scratch, scratch_bytes, s);
    return fmg_typed<float>(batch, nx, ny, hess, rhs, params, cycles, nit, u, has_initial, assume_initial_nonzero,
                            scratch, scratch_bytes, s);
}

int csg_dartel_expdef(int dtype, int batch, int nx, int ny, const void* velocity, int k, void* map_out, void* jac_out,
                      void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!velocity || !map_out || !scratch || k < 0 || k > 30)
        return csg::fail(CSG_ERR_ARG, "expdef: null pointer or bad k");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F64)
        return expdef_typed<double>(batch, nx, ny, velocity, k, map_out, jac_out, scratch, scratch_bytes, s);
    return expdef_typed<float>(batch, nx, ny, velocity, k, map_out, jac_out, scratch, scratch_bytes, s);
}

size_t csg_dartel_data_scratch_bytes(int dtype, int batch, int nx, int ny, int k, int checkpoint_every) {
    if (!check_dtype(dtype) || batch < 1 || nx < 1 || ny < 1 || k < 0 || k > 30 || checkpoint_every < 1) return 0;
    return dtype == CSG_DTYPE_F64 ? data_scratch<double>(batch, nx, ny, k, checkpoint_every)
                                  : data_scratch<float>(batch, nx, ny, k, checkpoint_every);
}

int csg_dartel_data_checkpoints(int k, int checkpoint_every) {
    if (k < 0 || k > 30 || checkpoint_every < 1) return 0;
    return data_checkpoints(k, checkpoint_every);
}

int csg_dartel_data_forward(int dtype, int batch, int nx, int ny, const void* velocity, const void* source,
                            const void* target, int k, int checkpoint_every, void* checkpoints, void* objective,
                            void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!velocity || !source || !target || !checkpoints || !objective || !scratch || k < 0 || k > 30 ||
        checkpoint_every < 1)
        return csg::fail(CSG_ERR_ARG, "data term forward: null pointer, bad k or checkpoint interval");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F64)
        return data_forward_typed<double>(batch, nx, ny, static_cast<const double*>(velocity),
                                          static_cast<const double*>(source), static_cast<const double*>(target), k,
                                          checkpoint_every, static_cast<double*>(checkpoints),
                                          static_cast<double*>(objective), scratch, scratch_bytes, s);
    return data_forward_typed<float>(batch, nx, ny, static_cast<const float*>(velocity),
                                     static_cast<const float*>(source), static_cast<const float*>(target), k,
                                     checkpoint_every, static_cast<float*>(checkpoints), static_cast<float*>(objective),
                                     scratch, scratch_bytes, s);
}

int csg_dartel_data_backward(int dtype, int batch, int nx, int ny, const void* source, const void* target, int k,
                             int checkpoint_every, const void* checkpoints, const void* grad_scale,
                             void* grad_velocity, void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    int rc = check_grid(dtype, batch, nx, ny);
    if (rc) return rc;
    if (!source || !target || !checkpoints || !grad_velocity || !scratch || k < 0 || k > 30 || checkpoint_every < 1)
        return csg::fail(CSG_ERR_ARG, "data term backward: null pointer, bad k or checkpoint interval");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F64)
        return data_backward_typed<double>(batch, nx, ny, static_cast<const double*>(source),
                                           static_cast<const double*>(target), k, checkpoint_every,
                                           static_cast<const double*>(checkpoints),
                                           static_cast<const double*>(grad_scale), static_cast<double*>(grad_velocity),
                                           scratch, scratch_bytes, s);
    return data_backward_typed<float>(batch, nx, ny, static_cast<const float*>(source),
                                      static_cast<const float*>(target), k, checkpoint_every,
                                      static_cast<const float*>(checkpoints), static_cast<const float*>(grad_scale),
                                      static_cast<float*>(grad_velocity), scratch, scratch_bytes, s);
}

}  // extern "C"
