// Final warp of SurfWarp on sm_100a: bilinear field sampling, application of
// a solved DARTEL flow to unit-sphere points, and the -avg blend of the x-
// and z-pole solutions.  One thread per point; float64 or float32 per the
// flow's dtype.  Compiled with --fmad=false; transcendental functions are
// CUDA's (their results differ from the reference's torch CPU ones by a few
// ulp, which the tests bound).
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/catsurf_b200.h"
#include "errors.h"

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

template <typename T>
struct Corners {
    int x0, x1, y0, y1;
    T dx1, dx2, dy1, dy2;
    __device__ __forceinline__ Corners(T x, T y, int nx, int ny) {
        const int ix = static_cast<int>(floor(x)), iy = static_cast<int>(floor(y));
        dx1 = x - static_cast<T>(ix);
        dy1 = y - static_cast<T>(iy);
        dx2 = T(1) - dx1;
        dy2 = T(1) - dy1;
        x0 = wrap_x(ix, nx);
        x1 = wrap_x(ix + 1, nx);
        y0 = reflect_y(iy, ny);
        y1 = reflect_y(iy + 1, ny);
    }
    template <typename F>
    __device__ __forceinline__ T bilinear(F f) const {
        return (f(x0, y0) * dx2 + f(x1, y0) * dx1) * dy2 + (f(x0, y1) * dx2 + f(x1, y1) * dx1) * dy1;
    }
};

// sample_field (dartel_grid.py:590-621).
template <typename T>
__global__ void k_sample(const T* __restrict__ field, int nx, int ny, int n, const T* __restrict__ xs,
                         const T* __restrict__ ys, T* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Corners<T> c(xs[i], ys[i], nx, ny);
    out[i] = c.bilinear([&](int x, int y) { return field[y * nx + x]; });
}

// _wrap_displacement (surface_warp.py:491-497).
template <typename T>
__device__ __forceinline__ T wrap_disp(T v) {
    if (v >= T(1)) v = v - floor(v);
    if (v <= T(-1)) v = v + floor(-v);
    if (v >= T(0.5)) v = v - T(1);
    if (v <= T(-0.5)) v = v + T(1);
    return v;
}

// apply_flow_to_sphere with unit-sphere points (surface_warp.py:500-584).
template <typename T>
__global__ void k_apply_flow(const float* __restrict__ points, int n, const T* __restrict__ flow, int nx, int ny,
                             int inverse, T* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T pi = T(3.141592653589793);
    const T x = static_cast<T>(points[3 * i]), y = static_cast<T>(points[3 * i + 1]);
    T z = static_cast<T>(points[3 * i + 2]);
    z = z < T(-1) ? T(-1) : (z > T(1) ? T(1) : z);
    const T theta0 = acos(z);
    T cw = -atan2(x, y);
    if (cw < T(0)) cw = cw + T(2.0 * 3.141592653589793);
    T u = (cw + T(3.141592653589793 / 2.0)) / T(2.0 * 3.141592653589793);
    if (u > T(1)) u = u - T(1);
    T v = theta0 / pi;
    const T gx = u * static_cast<T>(nx) - T(0.5);
    const T gy = v * static_cast<T>(ny) - T(0.5);
    const Corners<T> c(gx, gy, nx, ny);
    const int P = nx * ny;
    auto weight = [&](int row) { return sin(((static_cast<T>(row) + T(0.5)) / static_cast<T>(ny)) * pi); };
    const T su = c.bilinear([&](int col, int row) {
        return wrap_disp((flow[row * nx + col] - static_cast<T>(col) - T(1)) / static_cast<T>(nx)) * weight(row);
    });
    const T sv = c.bilinear([&](int col, int row) {
        return wrap_disp((flow[P + row * nx + col] - static_cast<T>(row) - T(1)) / static_cast<T>(ny)) * weight(row);
    });
    u = u + (inverse ? -su : su);
    v = v + (inverse ? -sv : sv);
    if (v < T(0)) u = u + T(0.5);
    if (v < T(0)) v = -v;
    if (v > T(1)) u = u + T(0.5);
    if (v > T(1)) v = T(2) - v;
    u = u - floor(u);
    v = v < T(0) ? T(0) : (v > T(1) ? T(1) : v);
    const T phi = u * T(2.0 * 3.141592653589793);
    const T theta = v * pi;
    const T st = sin(theta);
    const T wx = st * cos(phi), wy = st * sin(phi), wz = cos(theta);
    T norm = sqrt(wx * wx + wy * wy + wz * wz);
    const T eps = sizeof(T) == 8 ? T(2.220446049250313e-16) : T(1.1920928955078125e-07);
    norm = norm < eps ? eps : norm;
    out[3 * i] = wx / norm;
    out[3 * i + 1] = wy / norm;
    out[3 * i + 2] = wz / norm;
}

// _average_xz_surfaces (gpu_pipeline.py:248-271), float64 in, float32 out.
__global__ void k_average_xz(const double* __restrict__ xs, const double* __restrict__ zs, int n,
                             float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double pi = 3.141592653589793;
    auto clamp1 = [](double a) { return a < -1.0 ? -1.0 : (a > 1.0 ? 1.0 : a); };
    const double phx = acos(clamp1(xs[3 * i])) / pi;
    const double phz = acos(clamp1(zs[3 * i + 2])) / pi;
    const double ax = 2.0 * phx - 1.0, az = 2.0 * phz - 1.0;
    double wx = exp(-(ax * ax) / 0.1), wz = exp(-(az * az) / 0.1);
    wx = wx < 1e-19 ? 1e-19 : wx;
    wz = wz < 1e-19 ? 1e-19 : wz;
    const double total = wx + wz;
    double a[3];
    for (int k = 0; k < 3; ++k) a[k] = (wx * xs[3 * i + k] + wz * zs[3 * i + k]) / total;
    double norm = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    norm = norm < 2.220446049250313e-16 ? 2.220446049250313e-16 : norm;
    for (int k = 0; k < 3; ++k) out[3 * i + k] = static_cast<float>(a[k] / norm);
}

}  // namespace

extern "C" {

int csg_dartel_sample(int dtype, int nx, int ny, const void* field, int n, const void* x, const void* y, void* out,
                      csg_stream_t stream) {
    if ((dtype != CSG_DTYPE_F32 && dtype != CSG_DTYPE_F64) || nx < 1 || ny < 1 || n < 0 || !field ||
        (n > 0 && (!x || !y || !out)))
        return csg::fail(CSG_ERR_ARG, "sample_field: bad arguments");
    if (n == 0) return CSG_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned blocks = (n + kThreads - 1) / kThreads;
    if (dtype == CSG_DTYPE_F64)
        (csg::note_launch(), k_sample<double><<<blocks, kThreads, 0, s>>>(static_cast<const double*>(field), nx, ny, n,
                                                     static_cast<const double*>(x), static_cast<const double*>(y),
                                                     static_cast<double*>(out)));
    else
        (csg::note_launch(), k_sample<float><<<blocks, kThreads, 0, s>>>(static_cast<const float*>(field), nx, ny, n,
                                                    static_cast<const float*>(x), static_cast<const float*>(y),
                                                    static_cast<float*>(out)));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_apply_flow_to_sphere(int dtype, int n, const float* unit_points, int nx, int ny, const void* flow,
                             int inverse, void* out, csg_stream_t stream) {
    if ((dtype != CSG_DTYPE_F32 && dtype != CSG_DTYPE_F64) || nx < 1 || ny < 1 || n < 0 || !flow ||
        (n > 0 && (!unit_points || !out)))
        return csg::fail(CSG_ERR_ARG, "apply_flow_to_sphere: bad arguments");
    if (n == 0) return CSG_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned blocks = (n + kThreads - 1) / kThreads;
    if (dtype == CSG_DTYPE_F64)
        (csg::note_launch(), k_apply_flow<double><<<blocks, kThreads, 0, s>>>(unit_points, n, static_cast<const double*>(flow), nx, ny,
                                                         inverse, static_cast<double*>(out)));
    else
        (csg::note_launch(), k_apply_flow<float><<<blocks, kThreads, 0, s>>>(unit_points, n, static_cast<const float*>(flow), nx, ny, inverse,
                                                        static_cast<float*>(out)));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_average_xz(int n, const double* x_surface, const double* z_surface, float* out, csg_stream_t stream) {
    if (n < 0 || (n > 0 && (!x_surface || !z_surface || !out))) return csg::fail(CSG_ERR_ARG, "average_xz: bad arguments");
    if (n == 0) return CSG_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    (csg::note_launch(), k_average_xz<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(x_surface, z_surface, n, out));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

}  // extern "C"
