// flow.cu -- lattice-Boltzmann Stokes flow kernels (D2Q9 / D3Q19, TRT, Guo
// forcing, node bounce-back, periodic streaming) for sm_100a.
//
// What the reference does per iteration (prtlb_3d.py:427-445, prtlb_2d.py:449-474):
//   moments rho, u (u_x gets +g/2, u = 0 on solid)  -> feq
//   TRT collision (_trt_collide, prtlb_3d.py:142) + Guo term w_i(1-om-/2) 3 g e_ix
//   solid voxels: post-collision = the reversed ARRIVED populations
//   periodic streaming of every population (np.roll on every axis)
//
// Here one launch does one whole iteration in place, AA pattern:
//   even iteration: read f_i at the voxel, write the post-collision value
//                   into slot opp(i) of the same voxel;
//   odd iteration:  read f_i from slot opp(i) of voxel x - e_i, write the
//                   post-collision value into slot i of voxel x + e_i.
// With that pattern the reference's solid-voxel rule (reverse what arrived,
// then stream) is the identity on memory, so solid voxels are skipped and the
// transient, not only the steady state, is the reference's.
//
// Populations are stored shifted, h_i = f_i - w_i: in float32 the
// non-equilibrium part that carries the viscous stress is of the order of the
// force (1e-7) and would drown next to w_i ~ 0.3 (prtlb_2d.py:354-362).
#include <cuda_fp16.h>

#include "prt_internal.h"

namespace prt {

// -------------------------------------------------------------------------
// Lattices, in the storage frame (x, y, z).  The direction order and weights
// are the reference's (prtlb_3d.py:370-375, prtlb_2d.py:391-394); a D2Q9
// direction (ex, ey) is stored as (ex, 0, ey) because 2D grids are kept as
// (nx, 1, ny).
// -------------------------------------------------------------------------
struct D3Q19 {
    static constexpr int Q = 19;
    static constexpr int NP = 9;
    __host__ __device__ static constexpr int c(int i, int a) {
        return (a == 0) ? (i == 1 || i == 7 || i == 9 || i == 11 || i == 13   ? 1
                           : i == 2 || i == 8 || i == 10 || i == 12 || i == 14 ? -1
                                                                                : 0)
             : (a == 1) ? (i == 3 || i == 7 || i == 10 || i == 15 || i == 17   ? 1
                           : i == 4 || i == 8 || i == 9 || i == 16 || i == 18  ? -1
                                                                                : 0)
                        : (i == 5 || i == 11 || i == 14 || i == 15 || i == 18  ? 1
                           : i == 6 || i == 12 || i == 13 || i == 16 || i == 17 ? -1
                                                                                 : 0);
    }
    // pairs (a, b) with e_b = -e_a
    __host__ __device__ static constexpr int pa(int p) { return 2 * p + 1; }
    __host__ __device__ static constexpr int pb(int p) { return 2 * p + 2; }
    __host__ __device__ static constexpr int opp(int i) {
        return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1);
    }
    __host__ __device__ static constexpr double w(int i) {
        return i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    }
};

struct D2Q9 {
    static constexpr int Q = 9;
    static constexpr int NP = 4;
    // reference order: (0,0) (1,0) (0,1) (-1,0) (0,-1) (1,1) (-1,1) (-1,-1) (1,-1)
    __host__ __device__ static constexpr int ex(int i) {
        return (i == 1 || i == 5 || i == 8) ? 1 : ((i == 3 || i == 6 || i == 7) ? -1 : 0);
    }
    __host__ __device__ static constexpr int ey(int i) {
        return (i == 2 || i == 5 || i == 6) ? 1 : ((i == 4 || i == 7 || i == 8) ? -1 : 0);
    }
    __host__ __device__ static constexpr int c(int i, int a) {
        return a == 0 ? ex(i) : (a == 1 ? 0 : ey(i));
    }
    __host__ __device__ static constexpr int pa(int p) { return p < 2 ? p + 1 : p + 3; }
    __host__ __device__ static constexpr int pb(int p) { return p < 2 ? p + 3 : p + 5; }
    __host__ __device__ static constexpr int opp(int i) {
        return i == 0 ? 0 : (i < 5 ? ((i + 1) % 4) + 1 : ((i - 3) % 4) + 5);
    }
    __host__ __device__ static constexpr double w(int i) {
        return i == 0 ? 4.0 / 9.0 : (i < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
    }
};

// storage conversions ------------------------------------------------------
template <class S, class R>
struct Store;
template <>
struct Store<double, double> {
    __device__ static double ld(const double* p, float) { return *p; }
    __device__ static void st(double* p, double v, float) { *p = v; }
};
template <>
struct Store<float, float> {
    __device__ static float ld(const float* p, float) { return *p; }
    __device__ static void st(float* p, float v, float) { *p = v; }
};
template <>
struct Store<float, double> {  // float32 storage, float64 collision: only the store rounds
    __device__ static double ld(const float* p, float) { return (double)*p; }
    __device__ static void st(float* p, double v, float) { *p = (float)v; }
};
template <>
struct Store<__half, float> {
    __device__ static float ld(const __half* p, float inv) { return __half2float(*p) * inv; }
    __device__ static void st(__half* p, float v, float scale) {
        float s = v * scale;
        s = fminf(fmaxf(s, -65504.f), 65504.f);
        *p = __float2half_rn(s);
    }
};

struct Cell {
    int x, y, z;
    long long c;
    long long bx[3], by[3], bz[3];  // row bases for offsets -1, 0, +1 (periodic)
};

__device__ __forceinline__ Cell make_cell(long long c, const Grid& g) {
    Cell k;
    k.c = c;
    unsigned long long t = (unsigned long long)c;
    k.z = (int)(t % (unsigned)g.nz);
    t /= (unsigned)g.nz;
    k.y = (int)(t % (unsigned)g.ny);
    k.x = (int)(t / (unsigned)g.ny);
    const long long syz = (long long)g.ny * g.nz;
    int xm = k.x == 0 ? g.nx - 1 : k.x - 1, xp = k.x == g.nx - 1 ? 0 : k.x + 1;
    int ym = k.y == 0 ? g.ny - 1 : k.y - 1, yp = k.y == g.ny - 1 ? 0 : k.y + 1;
    int zm = k.z == 0 ? g.nz - 1 : k.z - 1, zp = k.z == g.nz - 1 ? 0 : k.z + 1;
    k.bx[0] = xm * syz; k.bx[1] = k.x * syz; k.bx[2] = xp * syz;
    k.by[0] = (long long)ym * g.nz; k.by[1] = (long long)k.y * g.nz; k.by[2] = (long long)yp * g.nz;
    k.bz[0] = zm; k.bz[1] = k.z; k.bz[2] = zp;
    return k;
}

// neighbour at offset (dx, dy, dz) in {-1, 0, 1}^3, periodic
__device__ __forceinline__ long long nbr(const Cell& k, int dx, int dy, int dz) {
    return k.bx[dx + 1] + k.by[dy + 1] + k.bz[dz + 1];
}

// Read the arrived populations of voxel k after `parity` AA half-steps.
template <class L, class S, class R, bool ODD>
__device__ __forceinline__ void load_arrived(const S* __restrict__ f, const Cell& k, long long N,
                                             float inv, R (&h)[L::Q]) {
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        if (!ODD) {
            h[i] = Store<S, R>::ld(f + (long long)i * N + k.c, inv);
        } else {
            long long src = nbr(k, -L::c(i, 0), -L::c(i, 1), -L::c(i, 2));
            h[i] = Store<S, R>::ld(f + (long long)L::opp(i) * N + src, inv);
        }
    }
}

template <class L, class R>
struct Moments {
    R drho, rho, ux, uy, uz;
};

template <class L, class R>
__device__ __forceinline__ Moments<L, R> moments(const R (&h)[L::Q], R half_g) {
    Moments<L, R> m;
    // density deviation, summed in pairs for accuracy
    R s = h[0];
#pragma unroll
    for (int p = 0; p < L::NP; ++p) s += (h[L::pa(p)] + h[L::pb(p)]);
    R jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
    for (int p = 0; p < L::NP; ++p) {
        const R d = h[L::pa(p)] - h[L::pb(p)];
        if (L::c(L::pa(p), 0) == 1) jx += d;
        if (L::c(L::pa(p), 0) == -1) jx -= d;
        if (L::c(L::pa(p), 1) == 1) jy += d;
        if (L::c(L::pa(p), 1) == -1) jy -= d;
        if (L::c(L::pa(p), 2) == 1) jz += d;
        if (L::c(L::pa(p), 2) == -1) jz -= d;
    }
    m.drho = s;
    m.rho = R(1) + s;
    m.ux = (jx + half_g) / m.rho;
    m.uy = jy / m.rho;
    m.uz = jz / m.rho;
    return m;
}

// TRT collision + Guo forcing in shifted variables; out[i] is the
// post-collision h of direction i.
template <class L, class R>
__device__ __forceinline__ void collide(const R (&h)[L::Q], const Moments<L, R>& m,
                                        const LbConst<R>& k, R (&out)[L::Q]) {
    const R usq = m.ux * m.ux + m.uy * m.uy + m.uz * m.uz;
    const R w0 = R(L::w(0));
    const R heq0 = w0 * (m.drho + m.rho * (R(-1.5) * usq));
    out[0] = h[0] - k.omp * (h[0] - heq0);
#pragma unroll
    for (int p = 0; p < L::NP; ++p) {
        const int a = L::pa(p), b = L::pb(p);
        const R wa = R(L::w(a));
        R eu = R(0);
        if (L::c(a, 0) == 1) eu += m.ux;
        if (L::c(a, 0) == -1) eu -= m.ux;
        if (L::c(a, 1) == 1) eu += m.uy;
        if (L::c(a, 1) == -1) eu -= m.uy;
        if (L::c(a, 2) == 1) eu += m.uz;
        if (L::c(a, 2) == -1) eu -= m.uz;
        const R heq_p = wa * (m.drho + m.rho * (R(4.5) * eu * eu - R(1.5) * usq));
        const R heq_m = wa * m.rho * (R(3) * eu);
        const R hp = R(0.5) * (h[a] + h[b]);
        const R hm = R(0.5) * (h[a] - h[b]);
        const R dp = k.omp * (hp - heq_p);
        const R dm = k.omm * (hm - heq_m);
        out[a] = h[a] - dp - dm + k.guo[p];
        out[b] = h[b] - dp + dm - k.guo[p];
    }
}

constexpr int kFlowThreads = 256;

template <class L, class S, class R, bool ODD, bool CHECK>
__global__ void __launch_bounds__(kFlowThreads) lb_step_kernel(S* __restrict__ f,
                                                                const uint8_t* __restrict__ fluid,
                                                                Grid g, LbConst<R> k,
                                                                const FlowCtrl* __restrict__ ctrl,
                                                                int kstep,
                                                                double* __restrict__ partials) {
    const long long it = ctrl->it_base + kstep;
    if (ctrl->done || it >= ctrl->nit) return;  // uniform over the grid
    const long long c = (long long)blockIdx.x * kFlowThreads + threadIdx.x;
    double acc = 0.0;
    if (c < g.n && fluid[c]) {
        const Cell cell = make_cell(c, g);
        R h[L::Q];
        load_arrived<L, S, R, ODD>(f, cell, g.n, k.inv_scale, h);
        const Moments<L, R> m = moments<L, R>(h, k.half_g);
        R out[L::Q];
        collide<L, R>(h, m, k, out);
#pragma unroll
        for (int i = 0; i < L::Q; ++i) {
            if (!ODD) {
                Store<S, R>::st(f + (long long)L::opp(i) * g.n + c, out[i], k.scale);
            } else {
                long long dst = nbr(cell, L::c(i, 0), L::c(i, 1), L::c(i, 2));
                Store<S, R>::st(f + (long long)i * g.n + dst, out[i], k.scale);
            }
        }
        if (CHECK) acc = fabs((double)m.ux);
    }
    if (CHECK) {
        __shared__ double sh[kFlowThreads / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x < 32) {
            double v = threadIdx.x < kFlowThreads / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (threadIdx.x == 0) partials[blockIdx.x] = v;
        }
    }
}

// Deterministic sum of per-block partials by one block.
__device__ double block_sum_fixed(const double* __restrict__ p, int n) {
    __shared__ double sh[256];
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

// FlowConvergence.done() at the end of a chunk of `every` iterations
// (prtlb_3d.py:220-235).  Also decides whether the while-graph goes on.
__global__ void flow_check_kernel(FlowCtrl* ctrl, const double* __restrict__ partials, int nb,
                                  cudaGraphConditionalHandle h, int use_handle) {
    const int done_before = ctrl->done;
    const long long base = ctrl->it_base;
    const long long end = min(base + (long long)ctrl->every, ctrl->nit);
    const bool full = (end - base) == ctrl->every;
    double s = 0.0;
    if (!done_before && full && ctrl->tol > 0) s = block_sum_fixed(partials, nb);
    if (threadIdx.x != 0) return;
    if (done_before) {
        if (use_handle) cudaGraphSetConditional(h, 0);
        return;
    }
    ctrl->iters = end;
    if (ctrl->tol > 0 && full && (end % ctrl->every) == 0) {
        const double u = ctrl->nfluid > 0 ? s / (double)ctrl->nfluid : 0.0;
        if (ctrl->has_prev) {
            ctrl->change = fabs(u - ctrl->prev) / fmax(fabs(u), 1e-30);
            if (ctrl->change <= ctrl->tol) ctrl->converged = 1;
        }
        ctrl->prev = u;
        ctrl->has_prev = 1;
    }
    ctrl->it_base = end;
    if (ctrl->converged || end >= ctrl->nit) ctrl->done = 1;
    if (use_handle) cudaGraphSetConditional(h, ctrl->done ? 0 : 1);
}

// Final field (prtlb_3d.py:451-456): v = (sum e f + g/2 x) / rho on pore
// voxels, 0 in solid, cast to float32; plus FP64 reductions used by the
// refusals of _checked_flow (prtlb_3d.py:267-316) and the permeability.
// partials layout: 5 doubles per block: sum ux, sum rho, sum speed, max speed, nonfinite
template <class L, class S, class R, bool ODD>
__global__ void __launch_bounds__(kFlowThreads) lb_moments_kernel(const S* __restrict__ f,
                                                                   const uint8_t* __restrict__ fluid,
                                                                   Grid g, LbConst<R> k,
                                                                   float* __restrict__ vel,
                                                                   double* __restrict__ partials) {
    const long long c = (long long)blockIdx.x * kFlowThreads + threadIdx.x;
    double sux = 0.0, srho = 0.0, ssp = 0.0, mx = 0.0, nonf = 0.0;
    if (c < g.n) {
        float vx = 0.f, vy = 0.f, vz = 0.f;
        if (fluid[c]) {
            const Cell cell = make_cell(c, g);
            R h[L::Q];
            load_arrived<L, S, R, ODD>(f, cell, g.n, k.inv_scale, h);
            const Moments<L, R> m = moments<L, R>(h, k.half_g);
            vx = (float)m.ux;
            vy = (float)m.uy;
            vz = (float)m.uz;
            sux = (double)m.ux;
            srho = (double)m.rho;
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

__global__ void fluid_mask_kernel(const uint8_t* __restrict__ mat, uint8_t* __restrict__ fluid,
                                  long long n, int pore) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) fluid[c] = (mat[c] == pore) ? 1 : 0;
}

// -------------------------------------------------------------------------
// launchers
// -------------------------------------------------------------------------
int flow_blocks(const Grid& g) { return (int)((g.n + kFlowThreads - 1) / kFlowThreads); }

template <class L, class S, class R>
static cudaError_t launch_step_t(bool odd, bool check, void* f, const uint8_t* fluid,
                                 const Grid& g, const void* kc, const FlowCtrl* ctrl, int kstep,
                                 double* partials, cudaStream_t s) {
    const LbConst<R>& k = *static_cast<const LbConst<R>*>(kc);
    dim3 grid(flow_blocks(g));
    S* fs = static_cast<S*>(f);
    if (!odd && !check) lb_step_kernel<L, S, R, false, false><<<grid, kFlowThreads, 0, s>>>(fs, fluid, g, k, ctrl, kstep, partials);
    if (!odd && check) lb_step_kernel<L, S, R, false, true><<<grid, kFlowThreads, 0, s>>>(fs, fluid, g, k, ctrl, kstep, partials);
    if (odd && !check) lb_step_kernel<L, S, R, true, false><<<grid, kFlowThreads, 0, s>>>(fs, fluid, g, k, ctrl, kstep, partials);
    if (odd && check) lb_step_kernel<L, S, R, true, true><<<grid, kFlowThreads, 0, s>>>(fs, fluid, g, k, ctrl, kstep, partials);
    return cudaGetLastError();
}

cudaError_t flow_launch_step(int nd, int precision, bool odd, bool check, void* f,
                             const uint8_t* fluid, const Grid& g, const void* kc,
                             const FlowCtrl* ctrl, int kstep, double* partials, cudaStream_t s) {
    if (nd == 3) {
        if (precision == PRT_FP64) return launch_step_t<D3Q19, double, double>(odd, check, f, fluid, g, kc, ctrl, kstep, partials, s);
        if (precision == PRT_FP32) return launch_step_t<D3Q19, float, double>(odd, check, f, fluid, g, kc, ctrl, kstep, partials, s);
        return launch_step_t<D3Q19, __half, float>(odd, check, f, fluid, g, kc, ctrl, kstep, partials, s);
    }
    if (precision == PRT_FP64) return launch_step_t<D2Q9, double, double>(odd, check, f, fluid, g, kc, ctrl, kstep, partials, s);
    if (precision == PRT_FP32) return launch_step_t<D2Q9, float, double>(odd, check, f, fluid, g, kc, ctrl, kstep, partials, s);
    return launch_step_t<D2Q9, __half, float>(odd, check, f, fluid, g, kc, ctrl, kstep, partials, s);
}

cudaError_t flow_launch_check(FlowCtrl* ctrl, const double* partials, int nblocks,
                              cudaGraphConditionalHandle h, int use_handle, cudaStream_t s) {
    flow_check_kernel<<<1, 256, 0, s>>>(ctrl, partials, nblocks, h, use_handle);
    return cudaGetLastError();
}

template <class L, class S, class R>
static cudaError_t launch_moments_t(bool odd, const void* f, const uint8_t* fluid, const Grid& g,
                                    const void* kc, float* vel, double* partials, cudaStream_t s) {
    const LbConst<R>& k = *static_cast<const LbConst<R>*>(kc);
    const S* fs = static_cast<const S*>(f);
    if (odd) lb_moments_kernel<L, S, R, true><<<flow_blocks(g), kFlowThreads, 0, s>>>(fs, fluid, g, k, vel, partials);
    else lb_moments_kernel<L, S, R, false><<<flow_blocks(g), kFlowThreads, 0, s>>>(fs, fluid, g, k, vel, partials);
    return cudaGetLastError();
}

cudaError_t flow_launch_moments(int nd, int precision, bool odd, const void* f,
                                const uint8_t* fluid, const Grid& g, const void* kc, float* vel,
                                double* partials, cudaStream_t s) {
    if (nd == 3) {
        if (precision == PRT_FP64) return launch_moments_t<D3Q19, double, double>(odd, f, fluid, g, kc, vel, partials, s);
        if (precision == PRT_FP32) return launch_moments_t<D3Q19, float, double>(odd, f, fluid, g, kc, vel, partials, s);
        return launch_moments_t<D3Q19, __half, float>(odd, f, fluid, g, kc, vel, partials, s);
    }
    if (precision == PRT_FP64) return launch_moments_t<D2Q9, double, double>(odd, f, fluid, g, kc, vel, partials, s);
    if (precision == PRT_FP32) return launch_moments_t<D2Q9, float, double>(odd, f, fluid, g, kc, vel, partials, s);
    return launch_moments_t<D2Q9, __half, float>(odd, f, fluid, g, kc, vel, partials, s);
}

cudaError_t flow_launch_fluid_mask(const uint8_t* mat, uint8_t* fluid, long long n, int pore,
                                   cudaStream_t s) {
    fluid_mask_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mat, fluid, n, pore);
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
