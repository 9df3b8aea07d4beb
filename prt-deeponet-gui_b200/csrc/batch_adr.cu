// batch_adr.cu -- the transport time loop of many solves per launch.
// Built with -fmad=false like adr.cu: the per-voxel step is adr_voxel, the
// check means are leaf_sum / tree_mean and the stop rule is adr_check, so a
// job's snapshots and step count are bit-identical to the single-solve loop.
//
// Per batch step: batch_adr_kernel advances every running job by one step
// (each at its own step count), batch_leaf_kernel forms the pairwise leaf
// sums of the jobs whose step is a check step, batch_ctrl_kernel finishes
// their trees, applies the stop rule and advances every job's step count.
#include "adr_core.cuh"

namespace prt {

namespace {
constexpr int kBatchAdrThreads = 256;
}

template <int ND, int NS>
__global__ void __launch_bounds__(kBatchAdrThreads)
    batch_adr_kernel(const AdrJob* __restrict__ jobs, const BatchTile* __restrict__ tiles,
                     const int* __restrict__ ntiles_p) {
    // the tile's job in shared memory: the per-voxel code reads its many
    // constants (feeds, diffusivities, rate constants) from there
    __shared__ __align__(16) AdrJob J;
    int t0, t1, cur = -1;
    tile_range(*ntiles_p, t0, t1);
    for (int t = t0; t < t1; ++t) {
        const BatchTile tl = tiles[t];
        if (tl.job != cur) {  // uniform over the block
            __syncthreads();  // the previous job's voxels are done with J
            block_copy(&J, jobs + tl.job);
            __syncthreads();
            cur = tl.job;
        }
        const AdrCtrl* ctrl = J.ctrl;
        if (ctrl->done) continue;
        const long long n = ctrl->n_base + 1;
        if (n > ctrl->limit) continue;
        // a job without biofilm takes the voxel step without the biofilm
        // selects (uniform over the block: J is the tile's job)
        const bool bf = J.d.has_bf != 0;
        for (int b = tl.b0; b < tl.b0 + tl.nb; ++b) {
            const long long kk = (long long)b * kBatchAdrThreads + threadIdx.x;
            if (kk < J.d.nm) {
                if (bf) adr_voxel<ND, NS, true>(J.d, J.p, n, kk);
                else adr_voxel<ND, NS, false>(J.d, J.p, n, kk);
            }
        }
    }
}

// A running job's step n = n_base + 1 just ran (*n_out is set whenever the
// job is not done); it is a check step when n is a multiple of `check` (the
// stop rule of prtlb_3d.py:1500-1548).
__device__ __forceinline__ bool adr_due(const AdrCtrl* c, long long* n_out) {
    if (c->done) return false;
    const long long n = c->n_base + 1;
    *n_out = n;
    return n <= c->limit && n % c->check == 0;
}

__global__ void __launch_bounds__(256)
    batch_leaf_kernel(const AdrJob* __restrict__ jobs, const LeafItem* __restrict__ items,
                      const int* __restrict__ nitems_p) {
    const int nitems = *nitems_p;
    for (int t = blockIdx.x; t < nitems; t += gridDim.x) {
        const LeafItem it = items[t];
        const AdrJob& J = jobs[it.job];
        long long n = 0;
        if (!adr_due(J.ctrl, &n)) continue;
        const int leaf = it.leaf0 + threadIdx.x;
        const PairTree& tr = J.d.tree;
        if (leaf >= tr.nleaf) continue;
        const float* src = J.d.buf[n & 1] + (long long)it.species * J.d.g.n;
        J.d.tree_vals[(long long)it.species * (tr.nleaf + tr.ninner) + leaf] =
            leaf_sum(src, J.d.idx, tr, leaf);
    }
}

__global__ void __launch_bounds__(256)
    batch_ctrl_kernel(const AdrJob* __restrict__ jobs, const int* __restrict__ njobs_p) {
    const int njobs = *njobs_p;
    for (int j = blockIdx.x; j < njobs; j += gridDim.x) {
        const AdrJob& J = jobs[j];
        AdrCtrl* ctrl = J.ctrl;
        long long n = 0;
        const bool skip = ctrl->done != 0;
        const bool due = !skip && adr_due(ctrl, &n);
        __syncthreads();  // every thread has read the control block before thread 0 writes it
        if (skip) continue;
        if (due) {
            const PairTree& tr = J.d.tree;
            for (int sp = 0; sp < ctrl->ns; ++sp)
                tree_mean(tr, J.d.nm, J.d.tree_vals + (long long)sp * (tr.nleaf + tr.ninner),
                          J.means + sp);
        }
        if (threadIdx.x == 0) {
            if (due) adr_check(ctrl, J.means, n, J.d.log, J.d.log_cap);
            ctrl->n_base = n;
            if (n >= ctrl->limit) ctrl->done = 1;
        }
        __syncthreads();
    }
}

template <int ND, int NS>
static cudaError_t launch_t(const AdrJob* jobs, const BatchTile* tiles, const int* ntiles, int grid,
                            cudaStream_t s) {
    batch_adr_kernel<ND, NS><<<grid, kBatchAdrThreads, 0, s>>>(jobs, tiles, ntiles);
    return cudaGetLastError();
}

template <int ND, int NS>
static int occ_t() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_adr_kernel<ND, NS>,
                                                      kBatchAdrThreads, 0) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return nb > 0 ? nb : 1;
}

#define PRT_NS_DISPATCH(FN, ND, ...)              \
    switch (ns) {                                 \
        case 1: return FN<ND, 1>(__VA_ARGS__);    \
        case 2: return FN<ND, 2>(__VA_ARGS__);    \
        case 3: return FN<ND, 3>(__VA_ARGS__);    \
        case 4: return FN<ND, 4>(__VA_ARGS__);    \
        case 5: return FN<ND, 5>(__VA_ARGS__);    \
        case 6: return FN<ND, 6>(__VA_ARGS__);    \
        case 7: return FN<ND, 7>(__VA_ARGS__);    \
        case 8: return FN<ND, 8>(__VA_ARGS__);    \
        default: break;                           \
    }

cudaError_t batch_launch_adr(int nd, int ns, const AdrJob* jobs, const BatchTile* tiles,
                             const int* ntiles, int grid, cudaStream_t s) {
    if (nd == 3) {
        PRT_NS_DISPATCH(launch_t, 3, jobs, tiles, ntiles, grid, s)
    } else {
        PRT_NS_DISPATCH(launch_t, 2, jobs, tiles, ntiles, grid, s)
    }
    return cudaErrorInvalidValue;
}

int batch_adr_occupancy(int nd, int ns) {
    if (nd == 3) {
        PRT_NS_DISPATCH(occ_t, 3)
    } else {
        PRT_NS_DISPATCH(occ_t, 2)
    }
    return 1;
}

cudaError_t batch_launch_adr_leaf(const AdrJob* jobs, const LeafItem* items, const int* nitems,
                                  int grid, cudaStream_t s) {
    batch_leaf_kernel<<<grid, 256, 0, s>>>(jobs, items, nitems);
    return cudaGetLastError();
}

cudaError_t batch_launch_adr_ctrl(const AdrJob* jobs, const int* njobs, int grid, cudaStream_t s) {
    batch_ctrl_kernel<<<grid, 256, 0, s>>>(jobs, njobs);
    return cudaGetLastError();
}

}  // namespace prt
