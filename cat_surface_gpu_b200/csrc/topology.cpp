// Host-side mesh topology and wavefront planning for the ordered
// Surf2Sphere sweeps.  Plain C++, no device memory.
#include <atomic>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/catsurf_b200.h"
#include "errors.h"

namespace {

int check_faces(int n_vertices, const int32_t* faces, int n_faces) {
    if (n_vertices < 1 || n_faces < 0 || (n_faces > 0 && faces == nullptr))
        return csg::fail(CSG_ERR_ARG, "mesh needs n_vertices >= 1 and a face array");
    for (int64_t i = 0; i < 3LL * n_faces; ++i)
        if (faces[i] < 0 || faces[i] >= n_vertices)
            return csg::fail(CSG_ERR_TOPOLOGY, "face index %d at position %lld is outside [0, %d)", faces[i],
                             static_cast<long long>(i), n_vertices);
    return CSG_OK;
}

void incidence(int n, const int32_t* faces, int n_faces, int32_t* off, int32_t* inc) {
    std::fill(off, off + n + 1, 0);
    for (int64_t i = 0; i < 3LL * n_faces; ++i) off[faces[i] + 1]++;
    for (int v = 0; v < n; ++v) off[v + 1] += off[v];
    std::vector<int32_t> fill(off, off + n);
    for (int f = 0; f < n_faces; ++f)
        for (int k = 0; k < 3; ++k) inc[fill[faces[3 * f + k]]++] = f;  // ascending face id
}

}  // namespace

namespace csg {
thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int fail(int code, const char* fmt, ...) {
    char buffer[1024];
    va_list args;
    va_start(args, fmt);
    std::vsnprintf(buffer, sizeof(buffer), fmt, args);
    va_end(args);
    g_last_error = buffer;
    return code;
}
}  // namespace csg

extern "C" {

const char* csg_last_error(void) { return csg::g_last_error.c_str(); }

int csg_abi_version(void) { return 3; }

long long csg_kernel_launches(void) { return csg::g_launches.load(std::memory_order_relaxed); }

int csg_mesh_incidence(int n_vertices, const int32_t* faces, int n_faces, int32_t* inc_off, int32_t* inc_face) {
    int rc = check_faces(n_vertices, faces, n_faces);
    if (rc) return rc;
    if (!inc_off || (n_faces > 0 && !inc_face)) return csg::fail(CSG_ERR_ARG, "null output");
    incidence(n_vertices, faces, n_faces, inc_off, inc_face);
    return CSG_OK;
}

int csg_mesh_neighbours(int n_vertices, const int32_t* faces, int n_faces, int32_t* nbr_off, int32_t* nbr,
                        int nbr_capacity) {
    int rc = check_faces(n_vertices, faces, n_faces);
    if (rc) return rc;
    if (!nbr_off) return csg::fail(CSG_ERR_ARG, "null output");
    // Directed edges of every triangle, then unique + sorted per source vertex.
    std::vector<int32_t> count(static_cast<size_t>(n_vertices) + 1, 0);
    for (int f = 0; f < n_faces; ++f)
        for (int k = 0; k < 3; ++k) count[faces[3 * f + k] + 1] += 2;
    for (int v = 0; v < n_vertices; ++v) count[v + 1] += count[v];
    std::vector<int32_t> raw(static_cast<size_t>(count[n_vertices]));
    std::vector<int32_t> fill(count.begin(), count.end() - 1);
    for (int f = 0; f < n_faces; ++f) {
        const int32_t* t = faces + 3 * f;
        for (int k = 0; k < 3; ++k) {
            int a = t[k], b = t[(k + 1) % 3], c = t[(k + 2) % 3];
            raw[fill[a]++] = b;
            raw[fill[a]++] = c;
        }
    }
    int64_t written = 0;
    nbr_off[0] = 0;
    for (int v = 0; v < n_vertices; ++v) {
        auto first = raw.begin() + count[v], last = raw.begin() + count[v + 1];
        std::sort(first, last);
        last = std::unique(first, last);
        // A face may repeat a vertex; a vertex is never its own neighbour.
        last = std::remove(first, last, v);
        int64_t m = last - first;
        if (nbr) {
            if (written + m > nbr_capacity) return csg::fail(CSG_ERR_ARG, "neighbour capacity too small");
            std::copy(first, last, nbr + written);
        }
        written += m;
        nbr_off[v + 1] = static_cast<int32_t>(written);
    }
    return static_cast<int>(written);
}

int csg_colour_groups(int n_vertices, const int32_t* nbr_off, const int32_t* nbr, int32_t* colour_off,
                      int32_t* members) {
    if (n_vertices < 1 || !nbr_off || !nbr || !colour_off || !members) return csg::fail(CSG_ERR_ARG, "bad arguments");
    // first fit in vertex order: the smallest colour no coloured neighbour has
    std::vector<int32_t> colour(static_cast<size_t>(n_vertices), -1);
    std::vector<int32_t> seen;  // seen[c] == v + 1: colour c is taken around v
    int n_colours = 0;
    for (int v = 0; v < n_vertices; ++v) {
        const int b = nbr_off[v], e = nbr_off[v + 1];
        if (b < 0 || e < b) return csg::fail(CSG_ERR_ARG, "neighbour offsets not ascending");
        for (int k = b; k < e; ++k) {
            const int w = nbr[k];
            if (w < 0 || w >= n_vertices) return csg::fail(CSG_ERR_TOPOLOGY, "neighbour index out of range");
            const int c = colour[w];
            if (c >= 0) {
                if (static_cast<size_t>(c) >= seen.size()) seen.resize(static_cast<size_t>(c) + 1, 0);
                seen[c] = v + 1;
            }
        }
        int c = 0;
        while (static_cast<size_t>(c) < seen.size() && seen[c] == v + 1) ++c;
        colour[v] = c;
        if (c + 1 > n_colours) n_colours = c + 1;
    }
    // members by colour, ascending within each colour (counting sort)
    std::fill(colour_off, colour_off + n_colours + 1, 0);
    for (int v = 0; v < n_vertices; ++v) colour_off[colour[v] + 1]++;
    for (int c = 0; c < n_colours; ++c) colour_off[c + 1] += colour_off[c];
    std::vector<int32_t> fill(colour_off, colour_off + n_colours);
    for (int v = 0; v < n_vertices; ++v) members[fill[colour[v]]++] = v;
    return n_colours;
}

int csg_normalise_sphere(int n_vertices, const float* in, float* out) {
    if (n_vertices < 1 || !in || !out) return csg::fail(CSG_ERR_ARG, "bad arguments");
    // centre: the sequential float64 sum of the float32 coordinates, divided by n
    double sum[3] = {0.0, 0.0, 0.0};
    for (int v = 0; v < n_vertices; ++v)
        for (int k = 0; k < 3; ++k) sum[k] = sum[k] + static_cast<double>(in[3LL * v + k]);
    double centre[3];
    for (int k = 0; k < 3; ++k) centre[k] = sum[k] / static_cast<double>(n_vertices);
    for (int v = 0; v < n_vertices; ++v) {
        double c[3];
        for (int k = 0; k < 3; ++k) c[k] = static_cast<double>(static_cast<float>(static_cast<double>(in[3LL * v + k]) - centre[k]));
        const double length = std::sqrt((c[0] * c[0] + c[1] * c[1]) + c[2] * c[2]);
        if (!std::isfinite(length) || length == 0.0) return csg::fail(CSG_ERR_ARG, "sphere vertex %d cannot be normalised", v);
        const double inv = 1.0 / length;
        for (int k = 0; k < 3; ++k) out[3LL * v + k] = static_cast<float>(c[k] * inv);
    }
    return CSG_OK;
}

int csg_dependency_levels(int n_vertices, const int32_t* nbr_off, const int32_t* nbr, int32_t* levels) {
    if (n_vertices < 1 || !nbr_off || !levels) return csg::fail(CSG_ERR_ARG, "bad arguments");
    int count = 0;
    for (int v = 0; v < n_vertices; ++v) {
        int level = 0;
        for (int k = nbr_off[v]; k < nbr_off[v + 1]; ++k) {
            int u = nbr[k];
            if (u < v) level = std::max(level, levels[u] + 1);
        }
        levels[v] = level;
        count = std::max(count, level + 1);
    }
    return count;
}

int csg_greedy_colours(int n_vertices, const int32_t* nbr_off, const int32_t* nbr, int32_t* colours) {
    if (n_vertices < 1 || !nbr_off || !colours) return csg::fail(CSG_ERR_ARG, "bad arguments");
    std::vector<int32_t> stamp;
    int n_colours = 0;
    for (int v = 0; v < n_vertices; ++v) colours[v] = -1;
    for (int v = 0; v < n_vertices; ++v) {
        int deg = nbr_off[v + 1] - nbr_off[v];
        if (static_cast<int>(stamp.size()) < deg + 2) stamp.resize(deg + 2, -1);
        for (int k = nbr_off[v]; k < nbr_off[v + 1]; ++k) {
            int c = colours[nbr[k]];
            if (c >= 0 && c <= deg) stamp[c] = v;
        }
        int colour = 0;
        while (stamp[colour] == v) ++colour;
        colours[v] = colour;
        n_colours = std::max(n_colours, colour + 1);
    }
    return n_colours;
}

int csg_areal_plan_build(int n_vertices, const int32_t* faces, int n_faces, int32_t* slot_off, int32_t* slot_tri,
                         int32_t* order, int32_t* level_begin, int32_t* level_end, csg_areal_plan_info* info) {
    int rc = check_faces(n_vertices, faces, n_faces);
    if (rc) return rc;
    if (!slot_off || !order || !level_begin || !level_end || !info || (n_faces > 0 && !slot_tri))
        return csg::fail(CSG_ERR_ARG, "null output");
    const int n = n_vertices;
    std::vector<int32_t> inc(static_cast<size_t>(3) * n_faces);
    incidence(n, faces, n_faces, slot_off, inc.data());
    int max_degree = 0;
    for (int v = 0; v < n; ++v) max_degree = std::max(max_degree, slot_off[v + 1] - slot_off[v]);
    for (int64_t s = 0; s < 3LL * n_faces; ++s) {
        const int32_t* t = faces + 3 * inc[s];
        slot_tri[4 * s + 0] = t[0];
        slot_tri[4 * s + 1] = t[1];
        slot_tri[4 * s + 2] = t[2];
        slot_tri[4 * s + 3] = inc[s];
    }
    // Unique lower and higher face neighbours of every vertex (the vertices a sweep
    // update reads), as two CSR arrays.  Each face neighbour of v appears in two of its
    // faces: a per-vertex stamp drops the repeats.  Their order does not matter: every
    // use below takes a maximum over them.
    std::vector<int32_t> lo_off(n + 1, 0), hi_off(n + 1, 0);
    std::vector<int32_t> lo_nb, hi_nb;
    lo_nb.reserve(static_cast<size_t>(3) * n_faces);
    hi_nb.reserve(static_cast<size_t>(3) * n_faces);
    {
        std::vector<int32_t> stamp(n, -1);
        for (int v = 0; v < n; ++v) {
            stamp[v] = v;
            for (int s = slot_off[v]; s < slot_off[v + 1]; ++s)
                for (int k = 0; k < 3; ++k) {
                    const int32_t u = slot_tri[4 * s + k];
                    if (stamp[u] != v) {
                        stamp[u] = v;
                        (u < v ? lo_nb : hi_nb).push_back(u);
                    }
                }
            lo_off[v + 1] = static_cast<int32_t>(lo_nb.size());
            hi_off[v + 1] = static_cast<int32_t>(hi_nb.size());
        }
    }
    // Levels: the longest chain of lower neighbours.
    std::vector<int32_t> levels(n, 0);
    int n_levels = 0;
    for (int v = 0; v < n; ++v) {
        int level = 0;
        for (int k = lo_off[v]; k < lo_off[v + 1]; ++k) level = std::max(level, levels[lo_nb[k]] + 1);
        levels[v] = level;
        n_levels = std::max(n_levels, level + 1);
    }
    int stride = 1;
    for (int v = 0; v < n; ++v)
        for (int k = hi_off[v]; k < hi_off[v + 1]; ++k) stride = std::max(stride, levels[hi_nb[k]] - levels[v] + 1);
    // Tighten the stride.  Any integer schedule f with 1 <= f(w) - f(v) <= D - 1
    // on every edge v < w runs vertex v of sweep s at step s D + f(v) with the
    // sequential read versions (lower neighbours this sweep, higher ones the
    // previous sweep).  The longest-path levels are one such f; the smallest
    // feasible D comes from difference constraints: lower D while the
    // relaxation f(w) >= f(v) + 1, f(v) >= f(w) - (D - 1) still converges
    // (a non-converging relaxation means a positive cycle, or too slow a
    // convergence to be worth it; both keep the last feasible D).
    {
        std::vector<int32_t> best = levels, f;
        std::vector<uint8_t> fwd_dirty(n), bwd_dirty(n);
        int last_iterations = 64;
        for (int trial = stride - 1; trial >= 2; --trial) {
            f = best;
            // feasible strides converge in a few relaxation sweeps (3 to 10 on
            // cortical hulls, each at most 5 more than the stride before it); a
            // stride that needs 8 more than the last one is treated as infeasible
            // -- only the schedule's length depends on it, and the infeasible
            // trial, which runs to the cap, is most of the planning time
            const int cap = std::min(4000, last_iterations + 8);
            bool converged = false;
            int it = 0;
            // Gauss-Seidel passes over a worklist: a vertex is evaluated only when a
            // neighbour its constraint reads changed since its last evaluation in that
            // pass direction (a clean vertex would keep its value), so every pass ends
            // with the values a full pass gives and the iteration counts are the same.
            // A forward pass only marks higher vertices (still ahead of it) and a
            // backward pass lower ones.  Byte flags measured faster than bitmaps scanned
            // by word (34 vs 38 ms on the 61k hull), and both than full passes (39 ms).
            std::fill(fwd_dirty.begin(), fwd_dirty.end(), 1);
            std::fill(bwd_dirty.begin(), bwd_dirty.end(), 1);
            for (; it < cap && !converged; ++it) {
                // In the forward pass no lower neighbour of v changes while v is
                // processed (and no higher one in the backward pass), so taking the
                // neighbours' maximum first raises f(v) exactly as one comparison per
                // neighbour would, without a branch per constraint.
                bool changed = false;
                int32_t* fv = f.data();
                for (int v = 0; v < n; ++v) {  // f(v) >= f(u) + 1 for lower neighbours u
                    if (!fwd_dirty[v]) continue;
                    fwd_dirty[v] = 0;
                    int32_t need = fv[v];
                    for (int k = lo_off[v]; k < lo_off[v + 1]; ++k) need = std::max(need, fv[lo_nb[k]] + 1);
                    if (need == fv[v]) continue;
                    fv[v] = need;
                    changed = true;
                    for (int k = hi_off[v]; k < hi_off[v + 1]; ++k) fwd_dirty[hi_nb[k]] = 1;  // later this pass
                    for (int k = lo_off[v]; k < lo_off[v + 1]; ++k) bwd_dirty[lo_nb[k]] = 1;
                }
                for (int v = n - 1; v >= 0; --v) {  // f(v) >= f(w) - (D - 1) for higher neighbours w
                    if (!bwd_dirty[v]) continue;
                    bwd_dirty[v] = 0;
                    int32_t need = fv[v];
                    for (int k = hi_off[v]; k < hi_off[v + 1]; ++k) need = std::max(need, fv[hi_nb[k]] - (trial - 1));
                    if (need == fv[v]) continue;
                    fv[v] = need;
                    changed = true;
                    for (int k = lo_off[v]; k < lo_off[v + 1]; ++k) bwd_dirty[lo_nb[k]] = 1;  // later this pass
                    for (int k = hi_off[v]; k < hi_off[v + 1]; ++k) fwd_dirty[hi_nb[k]] = 1;
                }
                converged = !changed;
            }
            if (!converged) break;
            const int32_t fmin = *std::min_element(f.begin(), f.end());
            const int32_t fmax = *std::max_element(f.begin(), f.end());
            if (fmax - fmin + 1 > n) break;  // level tables hold at most n levels
            for (int v = 0; v < n; ++v) f[v] -= fmin;
            best.swap(f);
            stride = trial;
            last_iterations = it;
        }
        levels.swap(best);
        n_levels = 0;
        for (int v = 0; v < n; ++v) n_levels = std::max(n_levels, levels[v] + 1);
    }
    // order: by (level mod stride, level, id) -- counting sort on level.
    std::vector<int32_t> per_level(static_cast<size_t>(n_levels) + 1, 0);
    for (int v = 0; v < n; ++v) per_level[levels[v] + 1]++;
    std::vector<int32_t> level_order;
    level_order.reserve(n_levels);
    for (int r = 0; r < stride; ++r)
        for (int l = r; l < n_levels; l += stride) level_order.push_back(l);
    int32_t cursor = 0;
    std::fill(level_begin, level_begin + n, 0);
    std::fill(level_end, level_end + n, 0);
    for (int l : level_order) {
        level_begin[l] = cursor;
        cursor += per_level[l + 1];
        level_end[l] = cursor;
    }
    std::vector<int32_t> fill(level_begin, level_begin + n_levels);
    for (int v = 0; v < n; ++v) order[fill[levels[v]]++] = v;
    info->n_vertices = n;
    info->n_faces = n_faces;
    info->n_levels = n_levels;
    info->level_stride = stride;
    info->max_degree = max_degree;
    info->n_slots = 3 * n_faces;
    return CSG_OK;
}

}  // extern "C"
