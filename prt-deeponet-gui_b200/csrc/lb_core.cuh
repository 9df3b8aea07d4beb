// lb_core.cuh -- lattices and the per-voxel TRT collision of the flow solve,
// shared by the single-solve and batched kernels.
#pragma once

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
// Pop<S>::H is the register type a stored population is held in; st() rounds
// the collision result to the storage type once.
template <class S>
struct Pop;
template <>
struct Pop<double> {
    using H = double;
    __device__ static double ld(const double* p, float) { return *p; }
    template <class R>
    __device__ static void st(double* p, R v, float) { *p = (double)v; }
};
template <>
struct Pop<float> {
    using H = float;
    __device__ static float ld(const float* p, float) { return *p; }
    template <class R>
    __device__ static void st(float* p, R v, float) { *p = (float)v; }
};
template <>
struct Pop<__half> {
    using H = float;
    __device__ static float ld(const __half* p, float inv) { return __half2float(*p) * inv; }
    template <class R>
    __device__ static void st(__half* p, R v, float scale) {
        float s = (float)v * scale;
        s = fminf(fmaxf(s, -65504.f), 65504.f);
        *p = __float2half_rn(s);
    }
};

// Precision modes: storage type S, arithmetic R for the symmetric part and
// RA for the momentum and the antisymmetric non-equilibrium part (a small
// difference of two O(u) numbers), and the resident blocks of kFlowThreads
// per SM the register budget is cut for (single-solve and batched steps).
// `staged`: the arrived populations go to shared memory by cp.async, so no
// register waits on a gather load (4- and 8-byte populations only).
struct ModeF64 {  // the reference's arithmetic
    using S = double;
    using R = double;
    using RA = double;
    static constexpr int min_blocks = 6;
    static constexpr int batch_min_blocks = 6;
    static constexpr bool staged = true;
};
struct ModeF32 {  // float32 populations, float32 collision
    using S = float;
    using R = float;
    using RA = float;
    // 64 registers (8 blocks per SM): at 48 (10 blocks) an iteration took
    // 5.46 us at 64^3 and 4.73 at 48^3, at 64 it takes 4.58 and 3.17
    static constexpr int min_blocks = 8;
    static constexpr int batch_min_blocks = 8;
    static constexpr bool staged = true;
};
struct ModeF32D {  // float32 populations, float64 momentum
    using S = float;
    using R = float;
    using RA = double;
    // 64 registers: at 48 (10 blocks) the step kernel spills, and 64^3
    // (917 blocks) still fits one wave at 8 blocks per SM (5.67 -> 5.41 us
    // per iteration; 128^3 unchanged)
    static constexpr int min_blocks = 8;
    static constexpr int batch_min_blocks = 8;
    static constexpr bool staged = true;
};
struct ModeF16 {  // scaled float16 populations, float32 collision
    using S = __half;
    using R = float;
    using RA = float;
    static constexpr int min_blocks = 6;
    static constexpr int batch_min_blocks = 6;
    static constexpr bool staged = false;
};

// Slots of the upstream voxels x - e_i of pore slot k (periodic), -1 where
// that voxel is rock.  The three candidate coordinates per axis are formed
// once; each direction then costs one index and one imap load.
template <class L>
__device__ __forceinline__ void upstream_slots(const FlowMap& fm, const Grid& g, int k,
                                               int (&src)[L::Q]) {
    int x, y, z;
    unpack_cell((unsigned)fm.cells[k], fm, x, y, z);
    const int X[3] = {x == 0 ? g.nx - 1 : x - 1, x, x == g.nx - 1 ? 0 : x + 1};
    const int Y[3] = {y == 0 ? g.ny - 1 : y - 1, y, y == g.ny - 1 ? 0 : y + 1};
    const int Z[3] = {z == 0 ? g.nz - 1 : z - 1, z, z == g.nz - 1 ? 0 : z + 1};
    src[0] = k;
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        const int a = 1 - L::c(i, 0), b = 1 - L::c(i, 1), c = 1 - L::c(i, 2);
        src[i] = fm.imap[(X[a] * g.ny + Y[b]) * g.nz + Z[c]];
    }
}

// Gather the arrived populations of pore voxel number k (see the file
// comment).  Lattices hold the pore voxels only, in C order: voxel
// cells[k] is slot k, and imap[voxel] is the slot of a pore voxel or -1.
// The two lattices of a solve as one array and 32-bit element offsets: the
// read lattice starts at element rd, the write lattice at wr (0 or Q*nf
// each; 2*Q*nf < 2^31 is checked at set-up), so every address is one
// 32-bit index and one wide multiply-add off the base.
template <class S>
struct Lat {
    S* f;
    int rd, wr, nf;
    __device__ const S* in(int i, int slot) const { return f + (rd + i * nf + slot); }
    __device__ S* out(int i, int slot) const { return f + (wr + i * nf + slot); }
};

template <class L, class S>
__device__ __forceinline__ Lat<S> lattices(S* f, int nf, bool odd) {
    const int qn = L::Q * nf;
    return Lat<S>{f, odd ? qn : 0, odd ? 0 : qn, nf};
}

// The element offsets (into the two lattices) of the populations slot k
// pulls in an iteration whose read lattice is `lat`: direction i from the
// upstream slot src[i] of the read lattice, or, when that voxel is rock,
// x's own value of two iterations back, opp(i) in the write lattice.
template <class L, class S>
__device__ __forceinline__ void pull_offsets(const Lat<S>& lat, int k, const int (&src)[L::Q],
                                             int (&off)[L::Q]) {
    off[0] = lat.rd + k;
#pragma unroll
    for (int i = 1; i < L::Q; ++i)
        off[i] = src[i] >= 0 ? lat.rd + i * lat.nf + src[i] : lat.wr + L::opp(i) * lat.nf + k;
}

// The same offsets from the pull tables fm.nbr, one per parity of the read
// lattice (coalesced: entry i-1 of every slot is one contiguous row).
template <class L, class S>
__device__ __forceinline__ void pull_offsets_table(const FlowMap& fm, const Lat<S>& lat, int k,
                                                   int (&off)[L::Q]) {
    const int* tab = fm.nbr + (lat.rd != 0 ? (L::Q - 1) * fm.nf : 0);
    off[0] = lat.rd + k;
#pragma unroll
    for (int i = 1; i < L::Q; ++i) off[i] = __ldg(tab + (i - 1) * fm.nf + k);
}

template <class L, class S>
__device__ __forceinline__ void gather_from_offsets(const Lat<S>& lat, const int (&off)[L::Q],
                                                    float inv, typename Pop<S>::H (&h)[L::Q]) {
#pragma unroll
    for (int i = 0; i < L::Q; ++i) h[i] = Pop<S>::ld(lat.f + off[i], inv);
}

template <class L, class S>
__device__ __forceinline__ void gather(const Lat<S>& lat, int k, const FlowMap& fm, const Grid& g,
                                       float inv, typename Pop<S>::H (&h)[L::Q]) {
    int src[L::Q], off[L::Q];
    upstream_slots<L>(fm, g, k, src);
    pull_offsets<L, S>(lat, k, src, off);
    gather_from_offsets<L, S>(lat, off, inv, h);
}

// 128-thread blocks: at 64^3 (458 blocks of 256 for 148 SMs) finer blocks
// balance the SMs better and cut an iteration from 6.25 to 5.73 us.
constexpr int kFlowThreads = 128;

// cp.async of one 4- or 8-byte population into this thread's shared slot.
template <class S>
__device__ __forceinline__ void cp_async_pop(S* dst, const S* src) {
    static_assert(sizeof(S) == 4 || sizeof(S) == 8, "cp.async copies 4 or 8 bytes here");
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (sizeof(S) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// The arrived populations of one thread in shared memory: element i of the
// thread's column (stride kFlowThreads).
template <class S>
struct Staged {
    const S* col;
    __device__ S operator[](int i) const { return col[i * kFlowThreads]; }
};

// The gather with the population loads issued as cp.async into `col` (this
// thread's column of a [Q][kFlowThreads] shared array): the same sources,
// but no register is held while a load is in flight.
template <class L, class S>
__device__ __forceinline__ void gather_staged(const Lat<S>& lat, const int (&off)[L::Q], S* col) {
#pragma unroll
    for (int i = 0; i < L::Q; ++i) cp_async_pop(col + i * kFlowThreads, lat.f + off[i]);
    cp_async_wait_all();
}

template <class R, class RA>
struct Moments {
    R drho, jsq;    // density deviation, rho u^2
    RA jx, jy, jz;  // J = rho u (with the half force on x)
    RA inv_rho;
};

// Moments of the arrived (shifted) populations (prtlb_3d.py:428-433):
// drho = sum h, J = rho u = sum e h + g/2 x.
template <class L, class R, class RA, class HA>
__device__ __forceinline__ Moments<R, RA> moments(const HA& h, double half_g) {
    Moments<R, RA> m;
    RA s = RA(h[0]);
    RA jx = RA(0), jy = RA(0), jz = RA(0);
#pragma unroll
    for (int p = 0; p < L::NP; ++p) {
        const int a = L::pa(p), b = L::pb(p);
        s += RA(h[a]) + RA(h[b]);
        const RA d = RA(h[a]) - RA(h[b]);
        if (L::c(a, 0) == 1) jx += d;
        if (L::c(a, 0) == -1) jx -= d;
        if (L::c(a, 1) == 1) jy += d;
        if (L::c(a, 1) == -1) jy -= d;
        if (L::c(a, 2) == 1) jz += d;
        if (L::c(a, 2) == -1) jz -= d;
    }
    jx += RA(half_g);
    m.jx = jx;
    m.jy = jy;
    m.jz = jz;
    const RA rho = RA(1) + s;
    m.inv_rho = RA(1) / rho;
    m.drho = R(s);
    m.jsq = R((jx * jx + jy * jy + jz * jz) * m.inv_rho);  // rho u^2 = |J|^2 / rho
    return m;
}

// TRT collision (_trt_collide, prtlb_3d.py:142-154) + Guo forcing in the
// shifted variables, written with J = rho u so that rho cancels in the
// antisymmetric equilibrium (w rho 3 e.u = 3 w e.J) and rho u u = J J / rho in
// the symmetric one.  The new population is h + delta with delta summed
// first, so the stored result rounds once; it goes to slot i of voxel c.
template <class L, class S, class R, class RA, class HA>
__device__ __forceinline__ void collide_store(const Lat<S>& lat, int c, const HA& h,
                                              const Moments<R, RA>& m, const LbParams& kc) {
    const R omp = R(kc.omp);
    const R inv_rho = R(m.inv_rho);
    const R heq0 = R(L::w(0)) * (m.drho - R(1.5) * m.jsq);
    const R h0 = R(h[0]);
    Pop<S>::st(lat.out(0, c), h0 - omp * (h0 - heq0), kc.scale);
#pragma unroll
    for (int p = 0; p < L::NP; ++p) {
        const int a = L::pa(p), b = L::pb(p);
        RA eJ = RA(0);
        if (L::c(a, 0) == 1) eJ += m.jx;
        if (L::c(a, 0) == -1) eJ -= m.jx;
        if (L::c(a, 1) == 1) eJ += m.jy;
        if (L::c(a, 1) == -1) eJ -= m.jy;
        if (L::c(a, 2) == 1) eJ += m.jz;
        if (L::c(a, 2) == -1) eJ -= m.jz;
        const R eJr = R(eJ);
        const R heq_p = R(L::w(a)) * (m.drho + (R(4.5) * eJr * eJr * inv_rho - R(1.5) * m.jsq));
        const R ha = R(h[a]), hb = R(h[b]);
        const R dp = omp * (R(0.5) * (ha + hb) - heq_p);
        const RA dma = RA(kc.omm) * (RA(0.5) * (RA(h[a]) - RA(h[b])) - RA(3.0 * L::w(a)) * eJ);
        const R dm = R(dma);
        const R gp = R(kc.guo[p]);
        Pop<S>::st(lat.out(a, c), ha + ((gp - dp) - dm), kc.scale);
        Pop<S>::st(lat.out(b, c), hb + ((dm - dp) - gp), kc.scale);
    }
}

// One pore voxel (slot k) of one LB iteration from the read lattice into
// the write lattice, the offsets of its pulls already found: gather,
// moments, collision, store; returns |u_x| for the convergence mean.
template <class L, class M>
__device__ __forceinline__ double lb_cell_offs(const Lat<typename M::S>& lat, const LbParams& kc,
                                               int k, const int (&off)[L::Q]) {
    using S = typename M::S;
    using R = typename M::R;
    using RA = typename M::RA;
    if constexpr (M::staged) {
        __shared__ S stage[L::Q * kFlowThreads];
        S* col = stage + threadIdx.x;
        gather_staged<L, S>(lat, off, col);
        const Staged<S> h{col};
        const Moments<R, RA> m = moments<L, R, RA>(h, kc.half_g);
        collide_store<L, S, R, RA>(lat, k, h, m, kc);
        return fabs((double)m.jx * (double)m.inv_rho);
    } else {
        typename Pop<S>::H h[L::Q];
        gather_from_offsets<L, S>(lat, off, kc.inv_scale, h);
        const Moments<R, RA> m = moments<L, R, RA>(h, kc.half_g);
        collide_store<L, S, R, RA>(lat, k, h, m, kc);
        return fabs((double)m.jx * (double)m.inv_rho);
    }
}

// The offsets of slot k's pulls: from the pull tables when the solve has
// them, else from the packed cell and the voxel map (the same offsets).
template <class L, class S>
__device__ __forceinline__ void find_pulls(const Lat<S>& lat, const FlowMap& fm, const Grid& g,
                                           int k, int (&off)[L::Q]) {
    if (fm.nbr) {
        pull_offsets_table<L, S>(fm, lat, k, off);
    } else {
        int src[L::Q];
        upstream_slots<L>(fm, g, k, src);
        pull_offsets<L, S>(lat, k, src, off);
    }
}

// The same, finding the pulls first.
template <class L, class M>
__device__ __forceinline__ double lb_cell_rw(const Lat<typename M::S>& lat, const FlowMap& fm,
                                             const Grid& g, const LbParams& kc, int k) {
    int off[L::Q];
    find_pulls<L, typename M::S>(lat, fm, g, k, off);
    return lb_cell_offs<L, M>(lat, kc, k, off);
}

// Block sum of one double per thread (warp shuffles, then the warp sums in
// order), stored by thread 0.  Both the single-solve and the batched step
// kernels reduce |u_x| with it, so their per-block partials agree bit for
// bit.  Every thread of the block must call it.
__device__ __forceinline__ void block_sum_store(double acc, double* out) {
    __shared__ double sh[kFlowThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < kFlowThreads / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) *out = v;
    }
    __syncthreads();
}

// Deterministic sum of n per-block partials by one block of kFlowThreads
// threads (fixed order: strided per thread, then a shared-memory tree).
// Loads bypass L1 because in the batched kernel other blocks of the same
// launch wrote the partials.
__device__ __forceinline__ double block_sum_fixed(const double* p, int n) {
    __shared__ double sh[kFlowThreads];
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += __ldcg(p + i);
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// FlowConvergence bookkeeping (prtlb_3d.py:220-235) once the iterations up
// to `end` are done; `sample` says whether the mean |u_x| of iteration end-1
// (sum s over the pore) was taken at this point (every `every` iterations).
// A sampled sum that is not finite stops the solve at once: the reference
// would run on to its cap (a NaN change never meets the tolerance) and then
// refuse the field, so stopping early changes only how long a doomed solve
// takes, never a finite result.
__device__ __forceinline__ void flow_ctrl_advance(FlowCtrl* c, long long end, bool sample,
                                                  double s) {
    c->iters = end;
    if (sample && !isfinite(s)) {
        c->nonfinite = 1;
    } else if (sample && c->tol > 0) {
        const double u = c->nfluid > 0 ? s / (double)c->nfluid : 0.0;
        if (c->has_prev) {
            c->change = fabs(u - c->prev) / fmax(fabs(u), 1e-30);
            if (c->change <= c->tol) c->converged = 1;
        }
        c->prev = u;
        c->has_prev = 1;
    }
    c->it_base = end;
    if (c->converged || c->nonfinite || end >= c->nit) c->done = 1;
}

}  // namespace prt
