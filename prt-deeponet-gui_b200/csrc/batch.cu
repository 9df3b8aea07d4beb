// batch.cu -- the flow time loop of many solves in one launch per iteration.
//
// A batch holds flow solves of any sizes; their pore slots are cut into
// blocks of kFlowThreads slots and listed as tiles (job, first block, block
// count).  One persistent launch walks the tile list and runs one LB iteration of every
// job that is not done, each job at its own iteration count and parity.
// The arithmetic per voxel is lb_cell_rw, the per-block |u_x| partials are
// block_sum_store over the same blocks of slots, and the convergence update is
// flow_ctrl_advance, so a job's iterations, decisions and final field are
// bit-identical to the single-solve loop whatever else shares the batch.
//
// A job's iteration count is implicit: the batch counts its steps on the
// device, and a job that joined when the batch had done s0 steps with c0
// iterations behind it is at c0 + (steps done) - s0 = (steps done) - g0.
// So the control block is written only when the iteration samples the
// convergence mean or reaches the cap: then every tile adds its block count
// to the job's arrival counter, and the tile that completes the count sums
// the partials, advances the control block (flow_ctrl_advance) and clears
// the counter.  Tiles of the same job read the control block before they
// arrive, so the update cannot race with them.
#include "lb_core.cuh"

namespace prt {

// UNI: every job of the launch has the constants `kcu` (the same force, tau
// and magic number), which the kernel then reads as a parameter, like the
// single-solve step, instead of from the job's descriptor in shared memory.
template <bool UNI>
__device__ __forceinline__ const LbParams& job_constants(const LbParams& kcu, const LbParams& own) {
    if constexpr (UNI) return kcu;
    else return own;
}

template <class L, class M, bool UNI>
__global__ void __launch_bounds__(kFlowThreads, M::batch_min_blocks)
    batch_flow_kernel(const FlowJob* __restrict__ jobs, const BatchTile* __restrict__ tiles,
                      const int* __restrict__ ntiles_p, const long long* __restrict__ gstep,
                      int k, LbParams kcu, int late) {
    using S = typename M::S;
    __shared__ int s_last;
    __shared__ __align__(16) FlowJob sj;  // the tile's job: constants read where they are used
    // programmatic dependent launch: the work list and the job descriptors
    // are not written inside the graph, so the first tile's descriptor is
    // copied while the previous step drains; control blocks and lattices
    // are touched only after griddepcontrol.wait; late: the next step is
    // let in after this one's work (see pdl_late)
    if (!late) griddep_launch_dependents();
    int t0, t1, cur = -1;
    tile_range(*ntiles_p, t0, t1);
    bool waited = false;
    long long done_steps = 0;  // batch steps done before this one
    for (int t = t0; t < t1; ++t) {
        const BatchTile tl = tiles[t];
        if (tl.job != cur) {  // uniform over the block
            block_copy(&sj, jobs + tl.job);
            cur = tl.job;
        }
        __syncthreads();
        if (!waited) {  // uniform over the block
            griddep_wait();
            waited = true;
            done_steps = __ldcg(gstep) + k;
        }
        FlowCtrl* ctrl = sj.ctrl;
        const long long it = done_steps - sj.g0;  // iterations done before this one
        const long long nit = __ldcg(&ctrl->nit);
        const bool run = !__ldcg(&ctrl->done) && it < nit;
        const bool check = ((it + 1) % __ldcg(&ctrl->every)) == 0;  // the sampled iterations
        const bool advance = check || it + 1 >= nit;
        if (!run) {  // uniform over the block
            __syncthreads();  // every thread has read ctrl before sj may change
            continue;
        }
        const int nf = sj.fm.nf;
        const Lat<S> lat = lattices<L>(static_cast<S*>(sj.f), nf, (it & 1) != 0);
#pragma unroll 1
        for (int b = tl.b0; b < tl.b0 + tl.nb; ++b) {
            const int slot = b * kFlowThreads + threadIdx.x;
            double acc = 0.0;
            if (slot < nf)
                acc = lb_cell_rw<L, M>(lat, sj.fm, sj.g, job_constants<UNI>(kcu, sj.kc), slot);
            if (check) block_sum_store(acc, sj.partials + b);
        }
        if (!advance) {  // uniform over the block
            __syncthreads();  // every thread is done with sj before it may change
            continue;
        }
        // every warp has read the control block and finished its voxels
        // before the tile arrives (the last arrival advances the block)
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();  // partials before the arrival
            const unsigned old = atomicAdd(sj.arrive, (unsigned)tl.nb);
            s_last = (old + (unsigned)tl.nb == (unsigned)sj.nb) ? 1 : 0;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            const double sum = check ? block_sum_fixed(sj.partials, sj.nb) : 0.0;
            if (threadIdx.x == 0) {
                flow_ctrl_advance(ctrl, it + 1, check, sum);
                *sj.arrive = 0u;
                __threadfence();
            }
        }
        __syncthreads();  // s_last and sj are reused by the next tile
    }
    if (late) griddep_launch_dependents();
}

template <class L, class M>
static int occupancy_t() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_flow_kernel<L, M, false>,
                                                      kFlowThreads, 0) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return nb > 0 ? nb : 1;
}

template <class L, class M>
static cudaError_t launch_batch_t(const FlowJob* jobs, const BatchTile* tiles, const int* ntiles,
                                  const long long* gstep, int k, const LbParams* uniform,
                                  int grid, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kFlowThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    // a batch step lets the next one in after its work whatever its grid:
    // its own pre-wait work is small (tile and descriptor), and 48 small
    // solves ran 56.9k solves/h with it against 52.3k with the release at
    // the start (one run each)
    const int late = pdl_late(true) ? 1 : 0;
    if (uniform)
        return cudaLaunchKernelEx(&cfg, batch_flow_kernel<L, M, true>, jobs, tiles, ntiles, gstep,
                                  k, *uniform, late);
    return cudaLaunchKernelEx(&cfg, batch_flow_kernel<L, M, false>, jobs, tiles, ntiles, gstep, k,
                              LbParams{}, late);
}


#define PRT_BATCH_DISPATCH(FN, ...)                                                  \
    if (nd == 3) {                                                                   \
        if (precision == PRT_FP64) return FN<D3Q19, ModeF64>(__VA_ARGS__);           \
        if (precision == PRT_FP32) return FN<D3Q19, ModeF32D>(__VA_ARGS__);          \
        if (precision == PRT_FP32_F32) return FN<D3Q19, ModeF32>(__VA_ARGS__);       \
        return FN<D3Q19, ModeF16>(__VA_ARGS__);                                      \
    }                                                                                \
    if (precision == PRT_FP64) return FN<D2Q9, ModeF64>(__VA_ARGS__);                \
    if (precision == PRT_FP32) return FN<D2Q9, ModeF32D>(__VA_ARGS__);               \
    if (precision == PRT_FP32_F32) return FN<D2Q9, ModeF32>(__VA_ARGS__);            \
    return FN<D2Q9, ModeF16>(__VA_ARGS__);

cudaError_t batch_launch_flow(int nd, int precision, const FlowJob* jobs, const BatchTile* tiles,
                              const int* ntiles, const long long* gstep, int k,
                              const LbParams* uniform, int grid, cudaStream_t s) {
    PRT_BATCH_DISPATCH(launch_batch_t, jobs, tiles, ntiles, gstep, k, uniform, grid, s)
}

__global__ void batch_gstep_kernel(long long* gstep, int k) { *gstep += k; }

cudaError_t batch_launch_gstep(long long* gstep, int k, cudaStream_t s) {
    batch_gstep_kernel<<<1, 1, 0, s>>>(gstep, k);
    return cudaGetLastError();
}

int batch_flow_occupancy(int nd, int precision) { PRT_BATCH_DISPATCH(occupancy_t) }

// out[i] = *done_ptrs[i]: the done flags of every job of a batch in one copy.
__global__ void batch_status_kernel(const int* const* __restrict__ done_ptrs, int n,
                                    int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = *done_ptrs[i];
}

cudaError_t batch_launch_status(const int* const* done_ptrs, int n, int* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    batch_status_kernel<<<(n + 255) / 256, 256, 0, s>>>(done_ptrs, n, out);
    return cudaGetLastError();
}

}  // namespace prt
