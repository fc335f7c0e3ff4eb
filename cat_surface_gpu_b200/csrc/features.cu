// Stencil feature operators of SurfWarp on sm_100a: barycentric resampling of
// a surface onto the stencil sphere, sheet mapping, iterative heat-kernel
// smoothing of geometry and of values, angle-weighted vertex normals,
// curvature types 5 and 2, and min-max normalisation.
//
// Follows src/cat_surface_gpu/surface_stencil.py:282-644.  Neighbour sums run
// over the unique, ascending 1-ring (CSR) in order -- the reference's padded
// neighbour table; normal accumulation per vertex runs corner 0 over all
// faces, then corner 1, then corner 2, each in face order -- the reference's
// three index_add_ calls.  Compiled with --fmad=false; acos / exp are CUDA's.
// Iterative smoothers run all their Jacobi iterations in one cooperative
// launch on the caller's stream (no host synchronisation inside): the grid
// strides over the points, a bounded grid barrier separates iterations, and
// the values ping-pong between two buffers.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/catsurf_b200.h"
#include "common.cuh"
#include "errors.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxSeries = 16;

struct SeriesParams {
    double sigma[kMaxSeries];
    int count[kMaxSeries];
};

inline unsigned blocks_for(long long n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ double norm3(double x, double y, double z) { return sqrt((x * x + y * y) + z * z); }
__device__ __forceinline__ float norm3f(float x, float y, float z) { return sqrtf((x * x + y * y) + z * z); }

// resample_vertices, float32 path (282-304): sum of float32-rounded float64 products.
__global__ void k_resample32(const float* __restrict__ v, const int* __restrict__ idx, const double* __restrict__ w,
                             int n, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; ++c) {
        float acc = 0.0f;
        for (int k = 0; k < 3; ++k) {
            const float term = static_cast<float>(static_cast<double>(v[3 * idx[3 * i + k] + c]) * w[3 * i + k]);
            acc = acc + term;
        }
        out[3 * i + c] = acc;
    }
}

// resample_vertices, float64 path (305-306).
__global__ void k_resample64(const double* __restrict__ v, const int* __restrict__ idx, const double* __restrict__ w,
                             int n, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; ++c) {
        const double a = v[3 * idx[3 * i] + c] * w[3 * i];
        const double b = v[3 * idx[3 * i + 1] + c] * w[3 * i + 1];
        const double d = v[3 * idx[3 * i + 2] + c] * w[3 * i + 2];
        out[3 * i + c] = (a + b) + d;
    }
}

// map_values_to_sheet (308-317).
__global__ void k_sheet(const double* __restrict__ values, const int* __restrict__ idx, const double* __restrict__ w,
                        int n, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (values[idx[3 * i]] * w[3 * i] + values[idx[3 * i + 1]] * w[3 * i + 1]) + values[idx[3 * i + 2]] * w[3 * i + 2];
}

// Per-block sums of the 3 F edge lengths (float64) for _edge_mean_distance (347-356).
template <typename T>
__global__ void k_edge_sum(const T* __restrict__ v, const int* __restrict__ faces, int n_faces,
                           double* __restrict__ partial) {
    __shared__ double buf[kThreads];
    const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    double len = 0.0;
    if (e < 3LL * n_faces) {
        const long long f = e / 3;
        const int k = static_cast<int>(e - 3 * f);
        const int a = faces[3 * f + k], b = faces[3 * f + (k + 1) % 3];
        len = norm3(static_cast<double>(v[3 * b]) - static_cast<double>(v[3 * a]),
                    static_cast<double>(v[3 * b + 1]) - static_cast<double>(v[3 * a + 1]),
                    static_cast<double>(v[3 * b + 2]) - static_cast<double>(v[3 * a + 2]));
    }
    buf[threadIdx.x] = len;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) buf[threadIdx.x] = buf[threadIdx.x] + buf[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = buf[0];
}

__global__ void k_sum_partials(const double* __restrict__ partial, int n, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = s + partial[i];
    out[0] = s;
}

// smooth_geometry (372-388), every iteration in one cooperative launch:
// float32 positions, float64 sums.  Iteration it reads `in` (it == 0) or the
// previous destination and writes `out` when an even number of iterations
// remain after it, else `tmp`, so the last lands in `out`; a grid barrier
// between iterations.
__global__ void k_smooth_geometry_all(const float* __restrict__ in, float* __restrict__ out, float* __restrict__ tmp,
                                      const int* __restrict__ off, const int* __restrict__ nbr, int n, int iterations,
                                      csg::Control* ctl, unsigned long long timeout_ns) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    unsigned int phase = 0;
    const float* src = in;
    for (int it = 0; it < iterations; ++it) {
        float* dst = ((iterations - 1 - it) % 2 == 0) ? out : tmp;
        for (int i = tid; i < n; i += nthreads) {
            const int b = off[i], e = off[i + 1];
            const double den = 1.0 + static_cast<double>(e - b) / 3.0;
            for (int c = 0; c < 3; ++c) {
                double sum = 0.0;
                for (int k = b; k < e; ++k) sum = sum + static_cast<double>(src[3 * nbr[k] + c]);
                const double num = static_cast<double>(src[3 * i + c]) + sum / 3.0;
                dst[3 * i + c] = static_cast<float>(num / den);
            }
        }
        if (it + 1 < iterations && csg::grid_barrier(ctl, phase, timeout_ns, it)) return;
        src = dst;
    }
}

// Heat weights of each (vertex, neighbour slot) for `series` sigmas and the
// per-vertex weight sums (390-476).  via_norm: distance through a norm then
// squared (smooth_values); else the squared components summed directly
// (smooth_values_many).
template <typename T>
__global__ void k_heat_weights(const T* __restrict__ geometry, const int* __restrict__ off, const int* __restrict__ nbr,
                               int n, SeriesParams sp, int series, int via_norm, double* __restrict__ weights,
                               double* __restrict__ wsum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (i >= n || s >= series) return;
    const int b = off[i], e = off[i + 1], slots = off[n];
    const double sig = sp.sigma[s];
    const double two = 2.0 * sig * sig;
    double total = 0.0;
    for (int k = b; k < e; ++k) {
        const int j = nbr[k];
        const double dx = static_cast<double>(geometry[3 * j]) - static_cast<double>(geometry[3 * i]);
        const double dy = static_cast<double>(geometry[3 * j + 1]) - static_cast<double>(geometry[3 * i + 1]);
        const double dz = static_cast<double>(geometry[3 * j + 2]) - static_cast<double>(geometry[3 * i + 2]);
        double dsq;
        if (via_norm) {
            const double d = norm3(dx, dy, dz);
            dsq = d * d;
        } else {
            dsq = (dx * dx + dy * dy) + dz * dz;
        }
        const double w = exp(-dsq / two);
        weights[static_cast<long long>(s) * slots + k] = w;
        total = total + w;
    }
    wsum[static_cast<long long>(s) * n + i] = total;
}

// smooth_values (390-476), every iteration of every series in one cooperative
// launch.  Series s reads in[s * stride ...] (stride 0 in the first iteration:
// every series starts from the caller's single value array) and writes
// out[s * n ...]; `in` and `out` never alias (Jacobi update); a series whose
// iteration count is reached copies its values through; a grid barrier
// between iterations.
__global__ void k_smooth_values_all(const double* __restrict__ in, double* __restrict__ out,
                                    double* __restrict__ tmp, const double* __restrict__ weights,
                                    const double* __restrict__ wsum, const int* __restrict__ off,
                                    const int* __restrict__ nbr, int n, int series, SeriesParams sp, int max_it,
                                    csg::Control* ctl, unsigned long long timeout_ns) {
    const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long nthreads = static_cast<long long>(gridDim.x) * blockDim.x;
    const int slots = off[n];
    unsigned int phase = 0;
    const double* src = in;
    long long stride = 0;
    for (int it = 0; it < max_it; ++it) {
        double* dst = ((max_it - 1 - it) % 2 == 0) ? out : tmp;
        for (long long q = tid; q < static_cast<long long>(series) * n; q += nthreads) {
            const int s = static_cast<int>(q / n), i = static_cast<int>(q - static_cast<long long>(s) * n);
            const long long base = static_cast<long long>(s) * n;
            const double* from = src + static_cast<long long>(s) * stride;
            if (it >= sp.count[s]) {
                dst[base + i] = from[i];
                continue;
            }
            const int b = off[i], e = off[i + 1];
            const double* w = weights + static_cast<long long>(s) * slots;
            double acc = 0.0;
            for (int k = b; k < e; ++k) acc = acc + w[k] * from[nbr[k]];
            dst[base + i] = (from[i] + acc) / (1.0 + wsum[base + i]);
        }
        if (it + 1 < max_it && csg::grid_barrier(ctl, phase, timeout_ns, it)) return;
        src = dst;
        stride = n;
    }
}

// Grid of a cooperative launch of `kernel`: as many kThreads-blocks as `work`
// needs, at most as many as the device holds at once.
int cooperative_grid(const void* kernel, long long work, unsigned* grid) {
    int device = 0, sms = 0, per_sm = 0;
    CSG_CUDA_CHECK(cudaGetDevice(&device));
    CSG_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CSG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0));
    const long long resident = static_cast<long long>(sms) * (per_sm > 0 ? per_sm : 1);
    *grid = static_cast<unsigned>(std::max(1LL, std::min(resident, (work + kThreads - 1) / kThreads)));
    return CSG_OK;
}

size_t align_up_256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Angle-weighted vertex normals (478-505).  inc lists (face << 2 | corner) per
// vertex sorted by (corner, face).
__global__ void k_vertex_normals(const float* __restrict__ v, const int* __restrict__ faces,
                                 const int* __restrict__ inc_off, const int* __restrict__ inc, int n,
                                 float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float eps = 1.1920928955078125e-07f;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int k = inc_off[i]; k < inc_off[i + 1]; ++k) {
        const int f = inc[k] >> 2, corner = inc[k] & 3;
        const int* t = faces + 3 * f;
        float p[3][3];
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) p[a][c] = v[3 * t[a] + c];
        float ea[3], eb[3], fn[3];
        for (int c = 0; c < 3; ++c) {
            ea[c] = p[1][c] - p[0][c];
            eb[c] = p[2][c] - p[0][c];
        }
        fn[0] = ea[1] * eb[2] - ea[2] * eb[1];
        fn[1] = ea[2] * eb[0] - ea[0] * eb[2];
        fn[2] = ea[0] * eb[1] - ea[1] * eb[0];
        float nn = norm3f(fn[0], fn[1], fn[2]);
        nn = nn < eps ? eps : nn;
        for (int c = 0; c < 3; ++c) fn[c] = fn[c] / nn;
        float prev[3], foll[3];
        const int pi = (corner + 2) % 3, fi = (corner + 1) % 3;
        for (int c = 0; c < 3; ++c) {
            prev[c] = p[pi][c] - p[corner][c];
            foll[c] = p[fi][c] - p[corner][c];
        }
        float den = norm3f(prev[0], prev[1], prev[2]) * norm3f(foll[0], foll[1], foll[2]);
        den = den < eps ? eps : den;
        float cosv = ((prev[0] * foll[0] + prev[1] * foll[1]) + prev[2] * foll[2]) / den;
        cosv = cosv < -1.0f ? -1.0f : (cosv > 1.0f ? 1.0f : cosv);
        const float angle = acosf(cosv);
        for (int c = 0; c < 3; ++c) acc[c] = acc[c] + fn[c] * angle;
    }
    float nn = norm3f(acc[0], acc[1], acc[2]);
    nn = nn < eps ? eps : nn;
    for (int c = 0; c < 3; ++c) out[3 * i + c] = acc[c] / nn;
}

// ((smoothed - geometry) . normals) in float32, widened to float64 (512-515).
__global__ void k_normal_displacement(const float* __restrict__ smoothed, const float* __restrict__ geometry,
                                      const float* __restrict__ normals, int n, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float d0 = smoothed[3 * i] - geometry[3 * i];
    const float d1 = smoothed[3 * i + 1] - geometry[3 * i + 1];
    const float d2 = smoothed[3 * i + 2] - geometry[3 * i + 2];
    out[i] = static_cast<double>((d0 * normals[3 * i] + d1 * normals[3 * i + 1]) + d2 * normals[3 * i + 2]);
}

// curvature_type2 point values before smoothing (552-615), float64.
__global__ void k_curvature2(const float* __restrict__ v, const float* __restrict__ normals, const int* __restrict__ off,
                             const int* __restrict__ nbr, int n, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = off[i], e = off[i + 1];
    auto dot = [](const double* a, const double* c) { return (a[0] * c[0] + a[1] * c[1]) + a[2] * c[2]; };
    double nm[3], p[3];
    for (int c = 0; c < 3; ++c) {
        nm[c] = static_cast<double>(normals[3 * i + c]);
        p[c] = static_cast<double>(v[3 * i + c]);
    }
    if (e - b < 1) {
        out[i] = 0.0;
        return;
    }
    double b0[3];
    {
        const int j = nbr[b];
        for (int c = 0; c < 3; ++c) b0[c] = static_cast<double>(v[3 * j + c]) - p[c];
        const double t = dot(b0, nm);
        for (int c = 0; c < 3; ++c) b0[c] = b0[c] - t * nm[c];
        double len = norm3(b0[0], b0[1], b0[2]);
        len = len < 2.220446049250313e-16 ? 2.220446049250313e-16 : len;
        for (int c = 0; c < 3; ++c) b0[c] = b0[c] / len;
    }
    const double mb[3] = {-b0[0], -b0[1], -b0[2]};
    const double b1[3] = {mb[1] * nm[2] - mb[2] * nm[1], mb[2] * nm[0] - mb[0] * nm[2], mb[0] * nm[1] - mb[1] * nm[0]};
    double s1 = 0.0, s2 = 0.0, s3 = 0.0, wx = 0.0, wy = 0.0, wxy = 0.0;
    for (int k = b; k < e; ++k) {
        const int j = nbr[k];
        double dc[3], dn[3];
        for (int c = 0; c < 3; ++c) {
            dc[c] = static_cast<double>(v[3 * j + c]) - p[c];
            dn[c] = static_cast<double>(normals[3 * j + c]) - nm[c];
        }
        const double tc = dot(dc, nm), tn = dot(dn, nm);
        double pc[3], pn[3];
        for (int c = 0; c < 3; ++c) {
            pc[c] = dc[c] - tc * nm[c];
            pn[c] = dn[c] - tn * nm[c];
        }
        const double dcx = dot(pc, b0), dcy = dot(pc, b1), dnx = dot(pn, b0), dny = dot(pn, b1);
        s1 = s1 + dcx * dnx * 1.0;
        s2 = s2 + (dcx * dny + dcy * dnx) * 1.0;
        s3 = s3 + dcy * dny * 1.0;
        wx = wx + dcx * dcx * 1.0;
        wy = wy + dcy * dcy * 1.0;
        wxy = wxy + dcx * dcy * 1.0;
    }
    const double wx2 = wx * wx, wy2 = wy * wy, wxy2 = wxy * wxy;
    const double den = (wx + wy) * (-wxy2 + wx * wy);
    const double safe = den != 0.0 ? den : 1.0;
    const double a = (s3 * wxy2 - s2 * wxy * wy + s1 * (-wxy2 + wx * wy + wy2)) / safe;
    const double bb = (-s3 * wx * wxy + s2 * wx * wy - s1 * wxy * wy) / safe;
    const double c = (-s2 * wx * wxy + s1 * wxy2 + s3 * (wx2 - wxy2 + wx * wy)) / safe;
    const double tr = a + c;
    const double det = a * c - bb * bb;
    double disc = tr * tr - 4.0 * det;
    disc = disc < 0.0 ? 0.0 : disc;
    const double root = sqrt(disc);
    const double k1 = (tr + root) / 2.0, k2 = (tr - root) / 2.0;
    out[i] = (e - b) > 2 ? sqrt((k1 * k1 + k2 * k2) / 2.0) : 0.0;
}

// Block min / max of `series` rows of n values, then normalisation.
__global__ void k_minmax_partial(const double* __restrict__ v, int n, double* __restrict__ partial) {
    __shared__ double mn[kThreads], mx[kThreads];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const long long base = static_cast<long long>(blockIdx.y) * n;
    const double x = i < n ? v[base + i] : INFINITY;
    mn[threadIdx.x] = x;
    mx[threadIdx.x] = i < n ? x : -INFINITY;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            mn[threadIdx.x] = fmin(mn[threadIdx.x], mn[threadIdx.x + s]);
            mx[threadIdx.x] = fmax(mx[threadIdx.x], mx[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * (static_cast<long long>(blockIdx.y) * gridDim.x + blockIdx.x)] = mn[0];
        partial[2 * (static_cast<long long>(blockIdx.y) * gridDim.x + blockIdx.x) + 1] = mx[0];
    }
}

__global__ void k_minmax_apply(const double* __restrict__ v, int n, const double* __restrict__ partial, int nblocks,
                               double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const long long base = static_cast<long long>(blockIdx.y) * n;
    __shared__ double lo, hi;
    if (threadIdx.x == 0) {
        double a = INFINITY, b = -INFINITY;
        for (int k = 0; k < nblocks; ++k) {
            a = fmin(a, partial[2 * (static_cast<long long>(blockIdx.y) * nblocks + k)]);
            b = fmax(b, partial[2 * (static_cast<long long>(blockIdx.y) * nblocks + k) + 1]);
        }
        lo = a;
        hi = b;
    }
    __syncthreads();
    if (i < n) out[base + i] = (v[base + i] - lo) / (hi - lo);
}

// True when byte ranges [a, a + na) and [b, b + nb) intersect.
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
    const auto pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    return pa < pb + nb && pb < pa + na;
}

}  // namespace

extern "C" {

int csg_feature_resample(int dtype, int n_out, const int32_t* indices, const double* weights, const void* vertices,
                         void* out, csg_stream_t stream) {
    if (n_out < 0 || (n_out > 0 && (!indices || !weights || !vertices || !out)) ||
        (dtype != CSG_DTYPE_F32 && dtype != CSG_DTYPE_F64))
        return csg::fail(CSG_ERR_ARG, "feature resample: bad arguments");
    if (n_out == 0) return CSG_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (dtype == CSG_DTYPE_F32)
        (csg::note_launch(), k_resample32<<<blocks_for(n_out), kThreads, 0, s>>>(static_cast<const float*>(vertices), indices, weights, n_out,
                                                           static_cast<float*>(out)));
    else
        (csg::note_launch(), k_resample64<<<blocks_for(n_out), kThreads, 0, s>>>(static_cast<const double*>(vertices), indices, weights,
                                                           n_out, static_cast<double*>(out)));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_feature_sheet_map(int n_cells, const int32_t* indices, const double* weights, const double* values,
                          double* out, csg_stream_t stream) {
    if (n_cells < 0 || (n_cells > 0 && (!indices || !weights || !values || !out)))
        return csg::fail(CSG_ERR_ARG, "sheet map: bad arguments");
    if (n_cells == 0) return CSG_OK;
    (csg::note_launch(), k_sheet<<<blocks_for(n_cells), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(values, indices, weights,
                                                                                        n_cells, out));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

size_t csg_feature_scratch_bytes(int n_points, int n_faces, int n_slots, int series) {
    if (n_points < 1 || n_faces < 0 || n_slots < 0 || series < 1) return 0;
    const size_t blocks_e = (3ULL * n_faces + kThreads - 1) / kThreads + 1;
    const size_t blocks_p = (static_cast<size_t>(n_points) + kThreads - 1) / kThreads + 1;
    size_t bytes = 0;
    bytes += 8 * blocks_e + 256;                                  // edge partials
    bytes += 12ULL * n_points + 256;                              // geometry ping-pong (float32)
    bytes += 8ULL * series * (n_slots + 2ULL * n_points) + 256;   // weights, weight sums, value ping-pong
    bytes += 16ULL * series * blocks_p + 256;                     // min / max partials
    return bytes + 1024;
}

int csg_feature_edge_sum(int dtype, int n_faces, const int32_t* faces, const void* vertices, double* out_sum,
                         void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    if (n_faces < 1 || !faces || !vertices || !out_sum || !scratch || (dtype != CSG_DTYPE_F32 && dtype != CSG_DTYPE_F64))
        return csg::fail(CSG_ERR_ARG, "edge sum: bad arguments");
    const unsigned nb = blocks_for(3LL * n_faces);
    if (scratch_bytes < 8ULL * nb) return csg::fail(CSG_ERR_ARG, "edge sum: scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    double* partial = static_cast<double*>(scratch);
    if (dtype == CSG_DTYPE_F32)
        (csg::note_launch(), k_edge_sum<float><<<nb, kThreads, 0, s>>>(static_cast<const float*>(vertices), faces, n_faces, partial));
    else
        (csg::note_launch(), k_edge_sum<double><<<nb, kThreads, 0, s>>>(static_cast<const double*>(vertices), faces, n_faces, partial));
    (csg::note_launch(), k_sum_partials<<<1, 32, 0, s>>>(partial, static_cast<int>(nb), out_sum));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_feature_smooth_geometry(int n_points, const int32_t* nbr_off, const int32_t* nbr, const float* vertices,
                                int iterations, float* out, void* scratch, size_t scratch_bytes, csg_stream_t stream) {
    if (n_points < 1 || !nbr_off || !nbr || !vertices || !out || iterations < 0 || !scratch)
        return csg::fail(CSG_ERR_ARG, "smooth geometry: bad arguments");
    const size_t control_at = align_up_256(12ULL * n_points);
    if (scratch_bytes < control_at + sizeof(csg::Control))
        return csg::fail(CSG_ERR_ARG, "smooth geometry: scratch too small");
    if (overlaps(vertices, 12ULL * n_points, out, 12ULL * n_points))
        return csg::fail(CSG_ERR_ARG, "smooth geometry: out must not overlap vertices");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    float* tmp = static_cast<float*>(scratch);
    if (iterations == 0) {
        CSG_CUDA_CHECK(cudaMemcpyAsync(out, vertices, 12ULL * n_points, cudaMemcpyDeviceToDevice, s));
        return CSG_OK;
    }
    // Ping-pong so that the last iteration lands in `out`; one cooperative launch.
    csg::Control* ctl = reinterpret_cast<csg::Control*>(static_cast<char*>(scratch) + control_at);
    CSG_CUDA_CHECK(cudaMemsetAsync(ctl, 0, sizeof(csg::Control), s));
    unsigned grid = 1;
    int rc = cooperative_grid(reinterpret_cast<const void*>(k_smooth_geometry_all), n_points, &grid);
    if (rc) return rc;
    unsigned long long timeout_ns = 2000000000ULL;
    const float* in = vertices;
    void* args[] = {&in, &out, &tmp, const_cast<int32_t**>(&nbr_off), const_cast<int32_t**>(&nbr), &n_points,
                    &iterations, &ctl, &timeout_ns};
    CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_smooth_geometry_all), dim3(grid),
                                               dim3(kThreads), args, 0, s));
    csg::note_launch();
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_feature_smooth_values(int n_points, const int32_t* nbr_off, const int32_t* nbr, int n_slots,
                              int geometry_dtype, const void* geometry, const double* values, int series,
                              const double* sigmas, const int32_t* iterations, int via_norm, double* out, void* scratch,
                              size_t scratch_bytes, csg_stream_t stream) {
    if (n_points < 1 || !nbr_off || !nbr || n_slots < 0 || !geometry || !values || series < 1 ||
        series > kMaxSeries || !sigmas || !iterations || !out || !scratch ||
        (geometry_dtype != CSG_DTYPE_F32 && geometry_dtype != CSG_DTYPE_F64))
        return csg::fail(CSG_ERR_ARG, "smooth values: bad arguments (1 <= series <= %d)", kMaxSeries);
    SeriesParams sp{};
    int max_it = 0;
    for (int k = 0; k < series; ++k) {
        sp.sigma[k] = sigmas[k];
        sp.count[k] = iterations[k];
        if (iterations[k] < 0) return csg::fail(CSG_ERR_ARG, "smooth values: negative iteration count");
        max_it = iterations[k] > max_it ? iterations[k] : max_it;
    }
    const size_t need = 8ULL * series * (static_cast<size_t>(n_slots) + 2ULL * n_points) + 1024;
    if (scratch_bytes < need) return csg::fail(CSG_ERR_ARG, "smooth values: scratch too small");
    if (overlaps(values, 8ULL * n_points, out, 8ULL * series * n_points))
        return csg::fail(CSG_ERR_ARG, "smooth values: out must not overlap values");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    double* weights = static_cast<double*>(scratch);
    double* wsum = weights + static_cast<size_t>(series) * n_slots;
    double* tmp = wsum + static_cast<size_t>(series) * n_points;
    const dim3 grid(blocks_for(n_points), series);
    if (geometry_dtype == CSG_DTYPE_F32)
        (csg::note_launch(), k_heat_weights<float><<<grid, kThreads, 0, s>>>(static_cast<const float*>(geometry), nbr_off, nbr, n_points, sp,
                                                         series, via_norm, weights, wsum));
    else
        (csg::note_launch(), k_heat_weights<double><<<grid, kThreads, 0, s>>>(static_cast<const double*>(geometry), nbr_off, nbr, n_points,
                                                          sp, series, via_norm, weights, wsum));
    // Ping-pong between `out` and `tmp` so that the last iteration lands in `out`;
    // the first iteration reads the caller's values directly; one cooperative launch.
    if (max_it > 0) {
        csg::Control* ctl = reinterpret_cast<csg::Control*>(
            static_cast<char*>(scratch) + align_up_256(8ULL * series * (static_cast<size_t>(n_slots) + 2ULL * n_points)));
        CSG_CUDA_CHECK(cudaMemsetAsync(ctl, 0, sizeof(csg::Control), s));
        unsigned cgrid = 1;
        int rc = cooperative_grid(reinterpret_cast<const void*>(k_smooth_values_all),
                                  static_cast<long long>(series) * n_points, &cgrid);
        if (rc) return rc;
        unsigned long long timeout_ns = 2000000000ULL;
        const double* in = values;
        void* args[] = {&in, &out, &tmp, &weights, &wsum, const_cast<int32_t**>(&nbr_off), const_cast<int32_t**>(&nbr),
                        &n_points, &series, &sp, &max_it, &ctl, &timeout_ns};
        CSG_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_smooth_values_all), dim3(cgrid),
                                                   dim3(kThreads), args, 0, s));
        csg::note_launch();
    }
    if (max_it == 0)
        for (int k = 0; k < series; ++k)
            CSG_CUDA_CHECK(cudaMemcpyAsync(out + static_cast<size_t>(k) * n_points, values, 8ULL * n_points,
                                           cudaMemcpyDeviceToDevice, s));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_feature_vertex_normals(int n_points, const int32_t* faces, const int32_t* inc_off, const int32_t* inc,
                               const float* vertices, float* out, csg_stream_t stream) {
    if (n_points < 1 || !faces || !inc_off || !inc || !vertices || !out)
        return csg::fail(CSG_ERR_ARG, "vertex normals: bad arguments");
    (csg::note_launch(), k_vertex_normals<<<blocks_for(n_points), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        vertices, faces, inc_off, inc, n_points, out));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_feature_normal_displacement(int n_points, const float* smoothed, const float* geometry, const float* normals,
                                    double* out, csg_stream_t stream) {
    if (n_points < 1 || !smoothed || !geometry || !normals || !out)
        return csg::fail(CSG_ERR_ARG, "normal displacement: bad arguments");
    (csg::note_launch(), k_normal_displacement<<<blocks_for(n_points), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        smoothed, geometry, normals, n_points, out));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_feature_curvature2(int n_points, const int32_t* nbr_off, const int32_t* nbr, const float* vertices,
                           const float* normals, double* out, csg_stream_t stream) {
    if (n_points < 1 || !nbr_off || !nbr || !vertices || !normals || !out)
        return csg::fail(CSG_ERR_ARG, "curvature type 2: bad arguments");
    (csg::note_launch(), k_curvature2<<<blocks_for(n_points), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        vertices, normals, nbr_off, nbr, n_points, out));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

int csg_feature_minmax(int n, int series, const double* values, double* out, void* scratch, size_t scratch_bytes,
                       csg_stream_t stream) {
    if (n < 1 || series < 1 || !values || !out || !scratch) return csg::fail(CSG_ERR_ARG, "minmax: bad arguments");
    const unsigned nb = blocks_for(n);
    if (scratch_bytes < 16ULL * nb * series) return csg::fail(CSG_ERR_ARG, "minmax: scratch too small");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    double* partial = static_cast<double*>(scratch);
    (csg::note_launch(), k_minmax_partial<<<dim3(nb, series), kThreads, 0, s>>>(values, n, partial));
    (csg::note_launch(), k_minmax_apply<<<dim3(nb, series), kThreads, 0, s>>>(values, n, partial, static_cast<int>(nb), out));
    CSG_CUDA_CHECK(cudaGetLastError());
    return CSG_OK;
}

}  // extern "C"
