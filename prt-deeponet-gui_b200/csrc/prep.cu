// prep.cu -- the walk from the inlet face through the pore space, for the
// geometry preparation done once per rock before its solves.
//
// What the reference does:
//   keep_inlet_connected (prtlb_3d.py:530-563): label the 6- (4-) connected
//     pore components with scipy, keep those touching the x = 0 face;
//   geodesic_steps (prt_core/conventions.py:72-115): a breadth-first walk
//     from the face, one Python queue step per voxel;
//   geodesic (build_practice_dataset.py:53-73): repeated relaxation sweeps
//     of d = min(d, neighbour + 1) until nothing changes.
// All three are one computation: the fewest face-neighbour steps from a pore
// voxel of the inlet face to every pore voxel (the reached set is exactly
// the union of the components touching the face).
//
// The same walk from any plane x_a = p (prt_walk_from_plane) serves the
// percolation checks of the dataset builders (build_dataset_3d.py:281-286,
// build_dataset_2d.py:290-294, build_geometry_3d.py:201-221): a component
// touches planes p and q exactly when the walk from p reaches plane q.
//
// Here the walk is level-synchronous and pulls: launch L visits every voxel
// once; a pore voxel not reached yet takes L + 1 if a face neighbour holds
// L.  A voxel is written only by its own thread, and during launch L the
// values change only from "unreached" to L + 1, neither of which is L, so
// the result does not depend on the order threads run in.  The host enqueues
// a chunk of levels and stops after the first chunk whose last level reached
// nothing new (no level can reach anything after one that reached nothing).
#include <vector>

#include "runtime_internal.h"

namespace prt {

namespace {

constexpr int kWalkThreads = 256;
constexpr int kUnreached = 0x7fffffff;
constexpr int kLevelsPerChunk = 32;

struct WalkGrid {
    Grid g;
    FastDiv dz, dy;
    int axis;   // storage axis of the seed plane (0 x, 1 y, 2 z)
    int plane;  // its coordinate along that axis
};

__device__ __forceinline__ void coords(unsigned c, const WalkGrid& w, int& x, int& y, int& z) {
    const unsigned q = fast_div(c, w.dz);
    z = (int)(c - q * w.dz.d);
    const unsigned xx = fast_div(q, w.dy);
    y = (int)(q - xx * w.dy.d);
    x = (int)xx;
}

// steps = 0 on the pore of the seed plane, unreached on the other pore,
// -1 elsewhere; counts[0] += pore voxels.
__global__ void __launch_bounds__(kWalkThreads)
    walk_init_kernel(const uint8_t* __restrict__ mat, WalkGrid w, int code, int* __restrict__ steps,
                     unsigned long long* __restrict__ counts) {
    const unsigned c = blockIdx.x * kWalkThreads + threadIdx.x;
    int pore = 0;
    if (c < (unsigned)w.g.n) {
        pore = mat[c] == code;
        int x, y, z;
        coords(c, w, x, y, z);
        const int along = w.axis == 0 ? x : (w.axis == 1 ? y : z);
        steps[c] = pore ? (along == w.plane ? 0 : kUnreached) : -1;
    }
    const int nb = __syncthreads_count(pore);
    if (threadIdx.x == 0 && nb) atomicAdd(counts, (unsigned long long)nb);
}

// One level: unreached pore voxels next to a voxel at `level` take level + 1;
// *flag = 1 when any did.
__global__ void __launch_bounds__(kWalkThreads)
    walk_level_kernel(int* __restrict__ steps, WalkGrid w, int level, int* __restrict__ flag) {
    const unsigned c = blockIdx.x * kWalkThreads + threadIdx.x;
    bool reached = false;
    if (c < (unsigned)w.g.n && steps[c] == kUnreached) {
        int x, y, z;
        coords(c, w, x, y, z);
        const int sz = 1, sy = w.g.nz, sx = w.g.ny * w.g.nz;
        bool hit = false;
        if (z > 0) hit |= steps[c - sz] == level;
        if (z < w.g.nz - 1) hit |= steps[c + sz] == level;
        if (y > 0) hit |= steps[c - sy] == level;
        if (y < w.g.ny - 1) hit |= steps[c + sy] == level;
        if (x > 0) hit |= steps[c - sx] == level;
        if (x < w.g.nx - 1) hit |= steps[c + sx] == level;
        if (hit) {
            steps[c] = level + 1;
            reached = true;
        }
    }
    if (__syncthreads_or(reached) && threadIdx.x == 0) *flag = 1;
}

// Unreached pore -> -2; counts[1] += reached pore voxels.
__global__ void __launch_bounds__(kWalkThreads)
    walk_final_kernel(int* __restrict__ steps, long long n, unsigned long long* __restrict__ counts) {
    const unsigned c = blockIdx.x * kWalkThreads + threadIdx.x;
    int reached = 0;
    if (c < (unsigned)n) {
        const int s = steps[c];
        if (s == kUnreached) steps[c] = -2;
        reached = s >= 0 && s != kUnreached;
    }
    const int nb = __syncthreads_count(reached);
    if (threadIdx.x == 0 && nb) atomicAdd(counts + 1, (unsigned long long)nb);
}

// label_materials (build_geometry_3d.py:224-239): pore 2, solid with a
// pore face neighbour 1, other solid 0; positions beyond the grid's faces
// count as solid (no wrap).  One thread per voxel, six neighbour reads
// through the cache; 2D grids are (nx, 1, ny).
__global__ void label_materials_kernel(const uint8_t* __restrict__ solid, WalkGrid w,
                                       uint8_t* __restrict__ out) {
    const long long n = w.g.n;
    const unsigned c = blockIdx.x * kWalkThreads + threadIdx.x;
    if (c >= (unsigned)n) return;
    if (!solid[c]) {
        out[c] = 2;
        return;
    }
    int x, y, z;
    coords(c, w, x, y, z);
    const Grid& g = w.g;
    const int sy = g.nz, sx = g.ny * g.nz;
    bool touch = false;
    if (x > 0) touch |= !solid[c - sx];
    if (x < g.nx - 1) touch |= !solid[c + sx];
    if (y > 0) touch |= !solid[c - sy];
    if (y < g.ny - 1) touch |= !solid[c + sy];
    if (z > 0) touch |= !solid[c - 1];
    if (z < g.nz - 1) touch |= !solid[c + 1];
    out[c] = touch ? 1 : 0;
}

}  // namespace

}  // namespace prt

using namespace prt;

extern "C" int prt_label_materials(prt_ctx* ctx, const uint8_t* solid, int32_t nd,
                                   const int32_t* dims, uint8_t* mat_out) {
    if (!ctx || !solid || !dims || !mat_out) return fail(ctx, PRT_E_INVALID, "null argument");
    if (nd != 2 && nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < nd; ++i)
        if (dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    const Grid g = make_grid(nd, dims);
    if (g.n >= (1ll << 31))
        return fail(ctx, PRT_E_INVALID, "grids of 2^31 voxels or more are not supported");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    PrepState& P = ctx->prep;
    CK(P.mat.ensure((size_t)g.n * 2));  // the solid grid, then the codes
    P.staged_mat = -1;
    uint8_t* d_solid = P.mat.as<uint8_t>();
    uint8_t* d_out = d_solid + g.n;
    CK(cudaMemcpyAsync(d_solid, solid, (size_t)g.n, cudaMemcpyHostToDevice, s));
    WalkGrid w;
    w.g = g;
    w.dz = make_fastdiv((unsigned)g.nz);
    w.dy = make_fastdiv((unsigned)g.ny);
    w.axis = 0;
    w.plane = 0;
    const unsigned nb = (unsigned)((g.n + kWalkThreads - 1) / kWalkThreads);
    label_materials_kernel<<<nb, kWalkThreads, 0, s>>>(d_solid, w, d_out);
    CK(cudaGetLastError());
    ctx->launches += 1;
    CK(cudaMemcpyAsync(mat_out, d_out, (size_t)g.n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return PRT_OK;
}

extern "C" int prt_walk_from_plane(prt_ctx* ctx, const uint8_t* mat, int32_t nd,
                                   const int32_t* dims, int32_t pore_code, int32_t axis,
                                   int32_t plane, int32_t* steps_out, int64_t* n_reached,
                                   int64_t* n_pore) {
    if (!ctx || !mat || !dims || !steps_out) return fail(ctx, PRT_E_INVALID, "null argument");
    if (nd != 2 && nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < nd; ++i)
        if (dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    if (axis < 0 || axis >= nd)
        return fail(ctx, PRT_E_INVALID, "the walk's axis must be one of the grid's axes");
    if (plane < 0 || plane >= dims[axis])
        return fail(ctx, PRT_E_INVALID, "the seed plane lies outside the grid");
    const Grid g = make_grid(nd, dims);
    // levels stay below the unreached marker: at most one per pore voxel,
    // plus one chunk
    if (g.n >= (1ll << 31) - 2 * kLevelsPerChunk)
        return fail(ctx, PRT_E_INVALID, "grids of 2^31 voxels or more are not supported");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    PrepState& P = ctx->prep;
    CK(P.mat.ensure((size_t)g.n));
    CK(P.steps.ensure((size_t)g.n * 4));
    CK(P.flags.ensure(kLevelsPerChunk * sizeof(int)));
    CK(P.counts.ensure(2 * sizeof(unsigned long long)));
    CK(cudaMemcpyAsync(P.mat.p, mat, (size_t)g.n, cudaMemcpyHostToDevice, s));
    P.staged_mat = -1;  // the buffer now holds the walk's grid
    CK(cudaMemsetAsync(P.counts.p, 0, 2 * sizeof(unsigned long long), s));
    WalkGrid w;
    w.g = g;
    w.dz = make_fastdiv((unsigned)g.nz);
    w.dy = make_fastdiv((unsigned)g.ny);
    w.axis = nd == 3 ? axis : (axis == 0 ? 0 : 2);  // 2D (nx, ny) is (nx, 1, ny)
    w.plane = plane;
    const unsigned nb = (unsigned)((g.n + kWalkThreads - 1) / kWalkThreads);
    int* steps = P.steps.as<int>();
    int* flags = P.flags.as<int>();
    unsigned long long* counts = P.counts.as<unsigned long long>();
    walk_init_kernel<<<nb, kWalkThreads, 0, s>>>(P.mat.as<uint8_t>(), w, pore_code, steps, counts);
    CK(cudaGetLastError());
    ctx->launches += 1;
    // at most one level per pore voxel, so the loop ends; in practice after
    // the longest shortest path
    std::vector<int> h(kLevelsPerChunk);
    for (long long base = 0; base <= g.n; base += kLevelsPerChunk) {
        CK(cudaMemsetAsync(flags, 0, kLevelsPerChunk * sizeof(int), s));
        for (int i = 0; i < kLevelsPerChunk; ++i)
            walk_level_kernel<<<nb, kWalkThreads, 0, s>>>(steps, w, (int)(base + i), flags + i);
        CK(cudaGetLastError());
        ctx->launches += kLevelsPerChunk;
        CK(cudaMemcpyAsync(h.data(), flags, kLevelsPerChunk * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (h[kLevelsPerChunk - 1] == 0) break;
    }
    walk_final_kernel<<<nb, kWalkThreads, 0, s>>>(steps, g.n, counts);
    CK(cudaGetLastError());
    ctx->launches += 1;
    unsigned long long hc[2];
    CK(cudaMemcpyAsync(steps_out, steps, (size_t)g.n * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (n_pore) *n_pore = (int64_t)hc[0];
    if (n_reached) *n_reached = (int64_t)hc[1];
    return PRT_OK;
}

extern "C" int prt_inlet_walk(prt_ctx* ctx, const uint8_t* mat, int32_t nd, const int32_t* dims,
                              int32_t pore_code, int32_t inlet_axis, int32_t* steps_out,
                              int64_t* n_reached, int64_t* n_pore) {
    return prt_walk_from_plane(ctx, mat, nd, dims, pore_code, inlet_axis, 0, steps_out, n_reached,
                               n_pore);
}
