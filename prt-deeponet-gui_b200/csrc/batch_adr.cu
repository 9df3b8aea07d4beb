// batch_adr.cu -- the transport time loop of many solves per launch.
// Built with -fmad=false like adr.cu: the per-voxel step is adr_voxel, the
// check means are the numpy pairwise leaves and tree_mean and the stop rule
// is adr_check, so a job's snapshots and step count are bit-identical to the
// single-solve loop.
//
// Per batch step one launch per class of jobs (dimension, chemicals) walks a
// work list of tiles of kBatchAdrBlock solute voxels and advances every
// running job by one step (each at its own step count, which is implicit:
// (batch steps done) - g0, see FlowJob).  On a job's check step its blocks
// also sum the pairwise-tree leaves of the new state (see AdrJob for the
// leaves that cross a block seam), and the block that completes the job's
// arrival count forms the means, applies the stop rule and writes the step
// count to the control block; on its last step (the step limit) the count
// is written the same way.  Other steps write nothing but the
// concentrations.  So a step is one launch per class, with no separate
// reduction or control launches.
#include "adr_core.cuh"

namespace prt {

namespace {
constexpr int kBatchAdrThreads = kBatchAdrBlock;
constexpr int kWarps = kBatchAdrThreads / 32;
// four resident blocks (64 registers): measured against 5, 6 and 8, which
// spill in the voxel step (32.1 against 33.8, 35.1 and 41.8 us a step for
// 48 small transport runs); without a bound the step takes 80-95 registers
constexpr int kBatchAdrMinBlocks = 4;
}

// leaf_sum of one leaf (at most 128 values) by one warp, with the same float
// additions in the same order: the lanes gather the values into `sh` (loads
// through L2: other blocks of the launch wrote some of them), lanes 0-7 run
// the eight interleaved accumulators and every lane then combines them and
// adds the tail.  The result is the same in every lane.
__device__ __forceinline__ float warp_leaf_sum(const float* __restrict__ s,
                                               const int* __restrict__ idx, int start, int len,
                                               float* sh) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < len; i += 32) sh[i] = __ldcg(s + idx[start + i]);
    __syncwarp();
    float res;
    if (len < 8) {
        res = 0.f;
        for (int i = 0; i < len; ++i) res = res + sh[i];
    } else {
        const int body = len - (len % 8);
        float r = 0.f;
        if (lane < 8) {
            r = sh[lane];
            for (int i = 8 + lane; i < body; i += 8) r = r + sh[i];
        }
        float q[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) q[k] = __shfl_sync(0xffffffffu, r, k);
        res = ((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]));
        for (int i = body; i < len; ++i) res = res + sh[i];
    }
    __syncwarp();  // sh is reused by the warp's next leaf
    return res;
}

// The leaves of block b of job J on a check step n, after the block's
// voxels of step n are stored: the leaves that start in the block and end
// inside it, plus each leaf across one of its two seams when the block is
// the second of the two blocks to get there.  Every thread of the block
// calls it.
// Not inlined, like job_step_end: the rare check-step code keeps its
// registers to itself, so the voxel step runs at the occupancy of its own
// register needs.
template <int NS>
__device__ __noinline__ void block_leaves(const AdrJob& J, int b, long long n, float (*sh)[128]) {
    __shared__ int s_lo, s_hi, s_l0, s_l1;
    const PairTree& tr = J.d.tree;
    if (threadIdx.x == 0) {
        const long long lo_at = (long long)b * kBatchAdrBlock;
        const long long hi_at = lo_at + kBatchAdrBlock;
        int l0 = J.blk_leaf[b], l1 = J.blk_leaf[b + 1];
        // a leaf started in block b - 1 that reaches into this block
        int lo = -1;
        if (b > 0 && l0 > 0 && tr.leaf_start[l0 - 1] + tr.leaf_len[l0 - 1] > lo_at) lo = l0 - 1;
        // this block's last leaf reaching into block b + 1
        int hi = -1;
        if (l1 > l0 && tr.leaf_start[l1 - 1] + tr.leaf_len[l1 - 1] > hi_at) {
            hi = l1 - 1;
            l1 -= 1;
        }
        if (lo >= 0 || hi >= 0) {
            __threadfence();  // this block's voxels before its seam arrivals
            if (lo >= 0) {
                if (atomicAdd(J.cnt + 1 + b, 1u) == 1u) J.cnt[1 + b] = 0u;  // second: ours
                else lo = -1;
            }
            if (hi >= 0) {
                if (atomicAdd(J.cnt + 2 + b, 1u) == 1u) J.cnt[2 + b] = 0u;
                else hi = -1;
            }
            __threadfence();  // the other block's voxels before the loads
        }
        s_lo = lo;
        s_hi = hi;
        s_l0 = l0;
        s_l1 = l1;
    }
    __syncthreads();
    const int l0 = s_l0, ninside = s_l1 - s_l0;
    const int nitems = ninside + (s_lo >= 0) + (s_hi >= 0);
    const int warp = threadIdx.x >> 5;
    const float* src = J.d.buf[n & 1];
    const long long N = J.d.g.n;
    for (int w = warp; w < nitems * NS; w += kWarps) {
        const int item = w / NS, sp = w % NS;
        int leaf;
        if (item < ninside) leaf = l0 + item;
        else if (item == ninside && s_lo >= 0) leaf = s_lo;
        else leaf = s_hi;
        const float v = warp_leaf_sum(src + (long long)sp * N, J.d.idx, tr.leaf_start[leaf],
                                      tr.leaf_len[leaf], sh[warp]);
        if ((threadIdx.x & 31) == 0)
            J.d.tree_vals[(long long)sp * (tr.nleaf + tr.ninner) + leaf] = v;
    }
    __syncthreads();  // s_* are reused by the block's next call
}

// The end of step n of job J by the block that completed its arrival count
// (every thread of the block calls it): on a check step the tree levels, the
// means and the stop rule; then the step count, the end at the limit, and
// the arrival counter cleared.
template <int NS>
__device__ __noinline__ void job_step_end(const AdrJob& J, long long n, long long limit, bool due) {
    __threadfence();
    AdrCtrl* ctrl = J.ctrl;
    if (due) {
        const PairTree& tr = J.d.tree;
        for (int sp = 0; sp < NS; ++sp)
            tree_mean<true>(tr, J.d.nm, J.d.tree_vals + (long long)sp * (tr.nleaf + tr.ninner),
                            J.means + sp);
    }
    if (threadIdx.x == 0) {
        if (due) adr_check(ctrl, J.means, n, J.d.log, J.d.log_cap);
        ctrl->n_base = n;
        if (n >= limit) ctrl->done = 1;
        J.cnt[0] = 0u;
        __threadfence();
    }
}

template <int ND, int NS>
__global__ void __launch_bounds__(kBatchAdrThreads, kBatchAdrMinBlocks)
    batch_adr_kernel(const AdrJob* __restrict__ jobs, const BatchTile* __restrict__ tiles,
                     const int* __restrict__ ntiles_p, const long long* __restrict__ gstep, int k,
                     int late) {
    // the tile's job in shared memory: the per-voxel code reads its many
    // constants (feeds, diffusivities, rate constants) from there
    __shared__ __align__(16) AdrJob J;
    __shared__ float sh[kWarps][128];
    __shared__ int s_last;
    // programmatic dependent launch: the work list and the job descriptors
    // are not written inside the graph, so the first tile's descriptor is
    // copied while the previous step drains; control blocks, counters and
    // concentrations are touched only after griddepcontrol.wait; late: the
    // next step is let in after this one's work (see pdl_late)
    if (!late) griddep_launch_dependents();
    int t0, t1, cur = -1;
    tile_range(*ntiles_p, t0, t1);
    bool waited = false;
    long long done_steps = 0;  // batch steps done before this one
    for (int t = t0; t < t1; ++t) {
        const BatchTile tl = tiles[t];
        if (tl.job != cur) {  // uniform over the block
            __syncthreads();  // the previous job's voxels are done with J
            block_copy(&J, jobs + tl.job);
            __syncthreads();
            cur = tl.job;
        }
        if (!waited) {
            griddep_wait();
            waited = true;
            done_steps = __ldcg(gstep) + k;
        }
        AdrCtrl* ctrl = J.ctrl;
        const int done = __ldcg(&ctrl->done);
        const long long n = done_steps - J.g0 + 1;  // the step this launch takes
        const long long limit = __ldcg(&ctrl->limit);
        const bool due = n % __ldcg(&ctrl->check) == 0;
        const bool advance = due || n >= limit;
        __syncthreads();  // every thread has read the control block
        if (done) continue;
        if (n > limit) {  // not reached: a run is marked done at its limit
            if (tl.b0 == 0 && threadIdx.x == 0) ctrl->done = 1;
            continue;
        }
        // a job without biofilm takes the voxel step without the biofilm
        // selects (uniform over the block: J is the tile's job)
        const bool bf = J.d.has_bf != 0;
        for (int b = tl.b0; b < tl.b0 + tl.nb; ++b) {
            const long long kk = (long long)b * kBatchAdrThreads + threadIdx.x;
            if (kk < J.d.nm) {
                if (bf) adr_voxel<ND, NS, true>(J.d, J.p, n, kk);
                else adr_voxel<ND, NS, false>(J.d, J.p, n, kk);
            }
            if (due) {
                __syncthreads();  // the block's voxels of step n are stored
                block_leaves<NS>(J, b, n, sh);
            }
        }
        if (!advance) continue;  // uniform; J changes only after a barrier
        // every thread has finished its voxels (and leaves) before the tile
        // arrives; the last arrival finishes the step of the job
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned old = atomicAdd(J.cnt, (unsigned)tl.nb);
            s_last = (old + (unsigned)tl.nb == (unsigned)J.nbk) ? 1 : 0;
        }
        __syncthreads();
        if (s_last) job_step_end<NS>(J, n, limit, due);  // uniform over the block
    }
    if (late) griddep_launch_dependents();
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

template <int ND, int NS>
static cudaError_t launch_t(const AdrJob* jobs, const BatchTile* tiles, const int* ntiles,
                            const long long* gstep, int k, int grid, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kBatchAdrThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    const int late = pdl_late(true) ? 1 : 0;  // as the batched flow step (batch.cu)
    return cudaLaunchKernelEx(&cfg, batch_adr_kernel<ND, NS>, jobs, tiles, ntiles, gstep, k, late);
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
                             const int* ntiles, const long long* gstep, int k, int grid,
                             cudaStream_t s) {
    if (nd == 3) {
        PRT_NS_DISPATCH(launch_t, 3, jobs, tiles, ntiles, gstep, k, grid, s)
    } else {
        PRT_NS_DISPATCH(launch_t, 2, jobs, tiles, ntiles, gstep, k, grid, s)
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

}  // namespace prt
