// lb_flow.cu -- lattice-Boltzmann Stokes flow kernels (D2Q9 / D3Q19, TRT, Guo
// forcing, node bounce-back, periodic streaming) for sm_100a.
//
// What the reference does per iteration (prtlb_3d.py:427-445, prtlb_2d.py:449-474):
//   moments rho, u (u_x gets +g/2, u = 0 on solid)  -> feq
//   TRT collision (_trt_collide, prtlb_3d.py:142) + Guo term w_i(1-om-/2) 3 g e_ix
//   solid voxels: post-collision = the reversed ARRIVED populations
//   periodic streaming of every population (np.roll on every axis)
//
// Here one launch does one whole iteration as a pull from lattice Lr (the
// post-collision populations of the previous iteration) into lattice Lw:
// a pore voxel x gathers f_i from x - e_i, collides and writes its values
// contiguously into its own slots of Lw.  When x - e_i is rock, the reference
// rule "the solid voxel sends back what arrived there one iteration earlier"
// makes the arriving value x's own post-collision population in direction
// opp(i) from two iterations ago -- which is still in Lw[opp(i)][x], not yet
// overwritten, and read by the same thread before it writes.  Solid voxels
// therefore do no work at all, and the transient is the reference's, not
// only its steady state.
//
// Populations are stored shifted, h_i = f_i - w_i: the non-equilibrium part
// that carries the viscous stress is of the order of the force (1e-7) and
// would drown next to w_i ~ 0.3 in float32 (prtlb_2d.py:354-362).
#include <cstdlib>

#include "lb_core.cuh"

namespace prt {

// One whole LB iteration t: lattice (t & 1) is read, lattice ((t + 1) & 1)
// written; solid voxels do nothing.  late: the next iteration is let in
// after this one's stores (see pdl_late).
template <class L, class M, bool ODD, bool CHECK>
__global__ void __launch_bounds__(kFlowThreads, M::min_blocks)
    lb_step_kernel(typename M::S* __restrict__ f, FlowMap fm, Grid g, LbParams kc,
                   const FlowCtrl* __restrict__ ctrl, int kstep, double* __restrict__ partials,
                   int late) {
    if (!late) griddep_launch_dependents();
    const int k = blockIdx.x * kFlowThreads + threadIdx.x;
    const Lat<typename M::S> lat = lattices<L>(f, fm.nf, ODD);
    // the pore maps never change during a solve: the pulls (with tables) or
    // the upstream slots (without) are looked up while the previous
    // iteration may still be running
    int off[L::Q], src[L::Q];
    if (k < fm.nf) {
        if (fm.nbr) pull_offsets_table<L>(fm, lat, k, off);
        else upstream_slots<L>(fm, g, k, src);
    }
    griddep_wait();
    const long long it = ctrl->it_base + kstep;
    if (ctrl->done || it >= ctrl->nit) return;  // uniform over the grid
    double acc = 0.0;
    if (k < fm.nf) {
        if (!fm.nbr) pull_offsets<L>(lat, k, src, off);
        const double ux = lb_cell_offs<L, M>(lat, kc, k, off);
        if (CHECK) acc = ux;
    }
    if (CHECK) block_sum_store(acc, partials + blockIdx.x);
    if (late) griddep_launch_dependents();
}

// FlowConvergence.done() at the end of a chunk of `every` iterations
// (prtlb_3d.py:220-235).  Also decides whether the while-graph goes on.
__global__ void flow_check_kernel(FlowCtrl* ctrl, const double* __restrict__ partials, int nb,
                                  cudaGraphConditionalHandle h, int use_handle) {
    const int done_before = ctrl->done;
    const long long base = ctrl->it_base;
    const long long end = min(base + (long long)ctrl->every, ctrl->nit);
    const bool full = (end - base) == ctrl->every;
    // the partials of the chunk's last iteration are summed at every full
    // chunk: for the convergence mean and the non-finite stop
    double s = 0.0;
    if (!done_before && full) s = block_sum_fixed(partials, nb);
    if (threadIdx.x != 0) return;
    if (done_before) {
        if (use_handle) cudaGraphSetConditional(h, 0);
        return;
    }
    flow_ctrl_advance(ctrl, end, full && (end % ctrl->every) == 0, s);
    if (use_handle) cudaGraphSetConditional(h, ctrl->done ? 0 : 1);
}

// Final field (prtlb_3d.py:451-456): v = (sum e f + g/2 x) / rho on pore
// voxels, 0 in solid, cast to float32; plus FP64 reductions used by the
// refusals of _checked_flow (prtlb_3d.py:267-316) and the permeability.
// The state after `iters` iterations is gathered exactly as iteration
// `iters` would gather it.
// partials layout: 5 doubles per block: sum ux, sum rho, sum speed, max speed, nonfinite
template <class L, class M, bool ODD>
__global__ void __launch_bounds__(kFlowThreads, M::min_blocks)
    lb_moments_kernel(const typename M::S* __restrict__ f, FlowMap fm, Grid g, LbParams k,
                      float* __restrict__ vel, double* __restrict__ partials) {
    using S = typename M::S;
    using R = typename M::R;
    using RA = typename M::RA;
    const int kk = blockIdx.x * kFlowThreads + threadIdx.x;
    const Lat<S> lat = lattices<L>(const_cast<S*>(f), fm.nf, ODD);
    double sux = 0.0, srho = 0.0, ssp = 0.0, mx = 0.0, nonf = 0.0;
    if (kk < fm.nf) {
        // solid voxels of vel were zeroed before this launch
        int cx, cy, cz;
        unpack_cell((unsigned)fm.cells[kk], fm, cx, cy, cz);
        const long long c = ((long long)cx * g.ny + cy) * g.nz + cz;
        float vx = 0.f, vy = 0.f, vz = 0.f;
        {
            typename Pop<S>::H h[L::Q];
            gather<L, S>(lat, kk, fm, g, k.inv_scale, h);
            const Moments<R, RA> m = moments<L, R, RA>(h, k.half_g);
            const RA ux = m.jx * m.inv_rho, uy = m.jy * m.inv_rho, uz = m.jz * m.inv_rho;
            vx = (float)ux;
            vy = (float)uy;
            vz = (float)uz;
            sux = (double)ux;
            srho = 1.0 + (double)m.drho;
            // speed the way _checked_flow computes it: float32, (x^2 + y^2) + z^2
            const float sp = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)),
                                             __fmul_rn(vz, vz)));
            nonf = (float)(!isfinite(vx)) + (float)(!isfinite(vy)) + (float)(!isfinite(vz));
            if (isfinite(sp)) {
                ssp = sp;
                mx = sp;
            }
        }
        // 2D grids: the reference returns (ux, uy, 0); our y is the storage z
        if (L::Q == 9) {
            vel[c] = vx;
            vel[g.n + c] = vz;
            vel[2 * g.n + c] = 0.f;
        } else {
            vel[c] = vx;
            vel[g.n + c] = vy;
            vel[2 * g.n + c] = vz;
        }
    }
    __shared__ double sh[5][kFlowThreads / 32];
    double v[5] = {sux, srho, ssp, mx, nonf};
#pragma unroll
    for (int q = 0; q < 5; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double t = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = (q == 3) ? fmax(v[q], t) : v[q] + t;
        }
        if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double t = threadIdx.x < kFlowThreads / 32 ? sh[q][threadIdx.x] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double u = __shfl_down_sync(0xffffffffu, t, o);
                t = (q == 3) ? fmax(t, u) : t + u;
            }
            if (threadIdx.x == 0) partials[(long long)blockIdx.x * 5 + q] = t;
        }
    }
}

__global__ void final_reduce_kernel(const double* __restrict__ partials, int nb, double* out) {
    __shared__ double sh[5][256];
    double v[5] = {0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double t = partials[(long long)i * 5 + q];
            v[q] = (q == 3) ? fmax(v[q], t) : v[q] + t;
        }
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) sh[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                double a = sh[q][threadIdx.x], b = sh[q][threadIdx.x + s];
                sh[q][threadIdx.x] = (q == 3) ? fmax(a, b) : a + b;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 5) out[threadIdx.x] = sh[threadIdx.x][0];
}

// Pore flags (set-up of the compacted layout).
__global__ void fluid_flag_kernel(const uint8_t* __restrict__ mat, long long n, int pore,
                                  uint8_t* __restrict__ flag) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) flag[c] = (mat[c] == pore) ? 1 : 0;
}

// imap[cells[k]] = k (imap was filled with -1 first).
// imap[cells[k]] = k (imap was filled with -1 first); then cells[k] is
// rewritten from the voxel index to the packed coordinates.
__global__ void imap_scatter_kernel(int* __restrict__ cells, int nf, int* __restrict__ imap,
                                    Grid g, int ys, int xs) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    const int v = cells[k];
    imap[v] = k;
    const int z = v % g.nz;
    const int t = v / g.nz;
    const int y = t % g.ny;
    const int x = t / g.ny;
    cells[k] = (int)(((unsigned)x << xs) | ((unsigned)y << ys) | (unsigned)z);
}

// The pull tables: for each parity p of the read lattice, nbr[p * (Q - 1) *
// nf + (i - 1) * nf + k] = the element offset slot k pulls direction i from.
template <class L>
__global__ void nbr_fill_kernel(FlowMap fm, Grid g, int* __restrict__ nbr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= fm.nf) return;
    int src[L::Q];
    upstream_slots<L>(fm, g, k, src);
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const Lat<char> lat = lattices<L, char>(nullptr, fm.nf, p != 0);
        int off[L::Q];
        pull_offsets<L, char>(lat, k, src, off);
        int* tab = nbr + p * (L::Q - 1) * fm.nf;
#pragma unroll
        for (int i = 1; i < L::Q; ++i) tab[(i - 1) * fm.nf + k] = off[i];
    }
}

// -------------------------------------------------------------------------
// launchers
// -------------------------------------------------------------------------
int flow_blocks(long long n) { return (int)((n + kFlowThreads - 1) / kFlowThreads); }

// Step kernels go out with programmatic stream serialisation (pdl_enabled,
// lb_core.cuh): kernel t+1 starts launching while kernel t drains, reads its
// upstream slots (the maps do not change during a solve) and waits in
// griddepcontrol.wait for t's results.  Measured on the B200 with 128-thread
// blocks: 64^3 float32 4.89 -> 4.82 us per iteration, float16 4.43 -> 4.18,
// 128^3 float32 41.3 -> 40.6.  A grid of one resident wave releases the
// next step only after its stores (pdl_late): 64^3 float32 collision
// 4.60 -> 4.09 us.

template <class L, class M, bool ODD, bool CHECK>
static cudaError_t launch_step_one(typename M::S* f, const FlowMap& fm, const Grid& g,
                                   const LbParams& k, const FlowCtrl* ctrl, int kstep,
                                   double* partials, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(flow_blocks(fm.nf));
    cfg.blockDim = dim3(kFlowThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    auto kern = lb_step_kernel<L, M, ODD, CHECK>;
    static const long long resident = [&] {
        int per_sm = 0, dev = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFlowThreads, 0) !=
                cudaSuccess ||
            cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            return 0ll;
        }
        return (long long)per_sm * sms;
    }();
    const int late = pdl_late(flow_blocks(fm.nf) <= resident) ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, f, fm, g, k, ctrl, kstep, partials, late);
}

template <class L, class M>
static cudaError_t launch_step_t(bool odd, bool check, void* f, const FlowMap& fm,
                                 const Grid& g, const LbParams& k, const FlowCtrl* ctrl, int kstep,
                                 double* partials, cudaStream_t s) {
    if (fm.nf <= 0) return cudaSuccess;
    typename M::S* fs = static_cast<typename M::S*>(f);
    if (!odd && !check) return launch_step_one<L, M, false, false>(fs, fm, g, k, ctrl, kstep, partials, s);
    if (!odd && check) return launch_step_one<L, M, false, true>(fs, fm, g, k, ctrl, kstep, partials, s);
    if (odd && !check) return launch_step_one<L, M, true, false>(fs, fm, g, k, ctrl, kstep, partials, s);
    return launch_step_one<L, M, true, true>(fs, fm, g, k, ctrl, kstep, partials, s);
}

#define PRT_DISPATCH(FN, ...)                                                        \
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

cudaError_t flow_launch_step(int nd, int precision, bool odd, bool check, void* f,
                             const FlowMap& fm, const Grid& g, const LbParams& k,
                             const FlowCtrl* ctrl, int kstep, double* partials, cudaStream_t s) {
    PRT_DISPATCH(launch_step_t, odd, check, f, fm, g, k, ctrl, kstep, partials, s)
}

cudaError_t flow_launch_check(FlowCtrl* ctrl, const double* partials, int nblocks,
                              cudaGraphConditionalHandle h, int use_handle, cudaStream_t s) {
    flow_check_kernel<<<1, kFlowThreads, 0, s>>>(ctrl, partials, nblocks, h, use_handle);
    return cudaGetLastError();
}

template <class L, class M>
static cudaError_t launch_moments_t(bool odd, const void* f, const FlowMap& fm, const Grid& g,
                                    const LbParams& k, float* vel, double* partials, cudaStream_t s) {
    if (fm.nf <= 0) return cudaSuccess;
    const typename M::S* fs = static_cast<const typename M::S*>(f);
    if (odd) lb_moments_kernel<L, M, true><<<flow_blocks(fm.nf), kFlowThreads, 0, s>>>(fs, fm, g, k, vel, partials);
    else lb_moments_kernel<L, M, false><<<flow_blocks(fm.nf), kFlowThreads, 0, s>>>(fs, fm, g, k, vel, partials);
    return cudaGetLastError();
}

cudaError_t flow_launch_moments(int nd, int precision, bool odd, const void* f,
                                const FlowMap& fm, const Grid& g, const LbParams& k, float* vel,
                                double* partials, cudaStream_t s) {
    PRT_DISPATCH(launch_moments_t, odd, f, fm, g, k, vel, partials, s)
}

cudaError_t flow_launch_flags(const uint8_t* mat, long long n, int pore, uint8_t* flag,
                              cudaStream_t s) {
    fluid_flag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mat, n, pore, flag);
    return cudaGetLastError();
}

cudaError_t flow_launch_imap(int* cells, int nf, int* imap, const Grid& g, int ys, int xs,
                             cudaStream_t s) {
    if (nf <= 0) return cudaSuccess;
    imap_scatter_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(cells, nf, imap, g, ys, xs);
    return cudaGetLastError();
}

cudaError_t flow_launch_nbr(int nd, const FlowMap& fm, const Grid& g, int* nbr, cudaStream_t s) {
    if (fm.nf <= 0) return cudaSuccess;
    const unsigned nb = (unsigned)((fm.nf + 255) / 256);
    if (nd == 3) nbr_fill_kernel<D3Q19><<<nb, 256, 0, s>>>(fm, g, nbr);
    else nbr_fill_kernel<D2Q9><<<nb, 256, 0, s>>>(fm, g, nbr);
    return cudaGetLastError();
}

cudaError_t flow_launch_final_reduce(const double* partials, int nb, double* out, cudaStream_t s) {
    final_reduce_kernel<<<1, 256, 0, s>>>(partials, nb, out);
    return cudaGetLastError();
}

// compile-time checks of the lattice tables
static_assert(D3Q19::opp(7) == 8 && D3Q19::opp(18) == 17, "D3Q19 opposites");
static_assert(D3Q19::c(13, 0) == 1 && D3Q19::c(13, 2) == -1, "D3Q19 e_13");
static_assert(D3Q19::c(18, 1) == -1 && D3Q19::c(18, 2) == 1, "D3Q19 e_18");
static_assert(D2Q9::pa(0) == 1 && D2Q9::pb(0) == 3 && D2Q9::pa(3) == 6 && D2Q9::pb(3) == 8, "D2Q9 pairs");
static_assert(D2Q9::opp(1) == 3 && D2Q9::opp(2) == 4 && D2Q9::opp(3) == 1 && D2Q9::opp(4) == 2 &&
                  D2Q9::opp(5) == 7 && D2Q9::opp(6) == 8 && D2Q9::opp(7) == 5 && D2Q9::opp(8) == 6,
              "D2Q9 opposites");
static_assert(D2Q9::ex(6) == -1 && D2Q9::ey(6) == 1 && D2Q9::ex(8) == 1 && D2Q9::ey(8) == -1, "D2Q9 e");

}  // namespace prt
