// adr_core.cuh -- per-voxel arithmetic of the transport step (solve_adr,
// prtlb_3d.py:1182-1413), shared by the single-solve and batched kernels.
// Every translation unit that includes it is compiled with -fmad=false: the
// reference integrates in float32 with numpy, one rounding per operation,
// and the operation order below is the reference's, so results are
// bit-identical to it.
#pragma once

#include "prt_internal.h"

namespace prt {

// numpy's elementwise semantics ---------------------------------------------
__device__ __forceinline__ float np_min(float a, float b) { return (a <= b || a != a) ? a : b; }
__device__ __forceinline__ float np_max(float a, float b) { return (a >= b || a != a) ? a : b; }

// min of two values that is NaN when either is (as np_min's value; the NaN
// may carry another payload).
__device__ __forceinline__ float min_nan(float a, float b) {
    float r;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// _muscl (prtlb_3d.py:650-705): up + 1/2 minmod(down - up, up - upup), the
// minmod written as 1/2 (sgn a + sgn b) min(|a|, |b|).  The signs are taken
// from the sign bits (copysign(1, d)), which differs from numpy's sign()
// only at d = +-0; there min(|a|, |b|) = 0, the slope is a zero of either
// sign, and up + 1/2 slope is up exactly unless up is -0.  No concentration
// is ever -0 (states start at +0 or above, a sum is -0 only of two -0
// operands, and the clip keeps its operand), so the result is numpy's bit
// for bit; NaN reaches it through the min.
__device__ __forceinline__ float muscl(float up, float upup, float down) {
    const float d1 = down - up;
    const float d2 = up - upup;
    const float slope =
        (0.5f * (copysignf(1.f, d1) + copysignf(1.f, d2))) * min_nan(fabsf(d1), fabsf(d2));
    return up + 0.5f * slope;
}

template <int ND>
struct Axes;
template <>
struct Axes<3> {
    static constexpr int n = 3;
    __host__ __device__ static constexpr int ax(int i) { return i; }
};
template <>
struct Axes<2> {  // a 2D grid (nx, ny) is stored as (nx, 1, ny)
    static constexpr int n = 2;
    __host__ __device__ static constexpr int ax(int i) { return i == 0 ? 0 : 2; }
};

// Index arithmetic is 32-bit: a transport grid holds fewer than 2^31
// values per buffer (ns x voxels, checked when the run begins).
struct VoxelPos {
    int p[3];
    int c;
};

// Coordinates of voxel c.
__device__ __forceinline__ VoxelPos voxel_pos(int c, const Grid& g) {
    VoxelPos v;
    v.c = c;
    unsigned t = (unsigned)c;
    v.p[2] = (int)(t % (unsigned)g.nz);
    t /= (unsigned)g.nz;
    v.p[1] = (int)(t % (unsigned)g.ny);
    v.p[0] = (int)(t / (unsigned)g.ny);
    return v;
}

// The same with the run's precomputed divisors (c < 2^31).
__device__ __forceinline__ VoxelPos voxel_pos(int c, const FastDiv& dz, const FastDiv& dy) {
    VoxelPos v;
    v.c = c;
    const unsigned t = (unsigned)c;
    const unsigned q = fast_div(t, dz);
    v.p[2] = (int)(t - q * dz.d);
    const unsigned x = fast_div(q, dy);
    v.p[1] = (int)(q - x * dy.d);
    v.p[0] = (int)x;
    return v;
}

// A load that is always issued, before the flags that decide whether its
// value is used are known: the address is in bounds either way (an
// edge-clamped neighbour), and the buffer is not written by this launch.
__device__ __forceinline__ float ld_early(const float* p) {
    float v;
    asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ int extent(const Grid& g, int a) {
    return a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
}
__device__ __forceinline__ int stride(const Grid& g, int a) {
    return a == 0 ? g.ny * g.nz : (a == 1 ? g.nz : 1);
}
// index of the low face of voxel v along axis a in the (n_a + 1)-long face array
__device__ __forceinline__ int face_lo(const Grid& g, const VoxelPos& v, int a) {
    if (a == 0) return v.c;
    if (a == 1) return (v.p[0] * (g.ny + 1) + v.p[1]) * g.nz + v.p[2];
    return (v.p[0] * g.ny + v.p[1]) * (g.nz + 1) + v.p[2];
}
__device__ __forceinline__ int face_step(const Grid& g, int a) {
    return a == 0 ? g.ny * g.nz : (a == 1 ? g.nz : 1);
}

// A neighbour value of chemical j.  Every neighbour that is actually read is a
// solute voxel (the open / far flags guarantee it), so it is on the inlet
// plane exactly when its x is 0; there the pinned feed replaces the stored
// value (step(), prtlb_3d.py:1392-1400, pins before transport).
__device__ __forceinline__ float ld_c(const float* __restrict__ Cj, int c, int x, bool pin,
                                      float feed) {
    const float v = ld_early(Cj + c);
    return (pin && x == 0) ? feed : v;
}

// One axis of transport() at one voxel (prtlb_3d.py:1182-1208), from the
// four neighbour values along the axis (clamped positions, inlet feed already
// applied), the two face velocities and the voxel's flags: adds the axis'
// diffusion and advection to `out` and its velocity difference to `divu`, in
// the reference's operation order.  BF: the run has biofilm; without it no
// voxel carries a biofilm flag, every face takes the pore diffusivity, and
// the biofilm count is not formed.  Every transport kernel calls this, so
// they compute the same function bit for bit.
template <bool BF>
__device__ __forceinline__ void transport_axis(float& out, float& divu, float Cc, float vm1,
                                               float vm2, float vp1, float vp2, float uL,
                                               float uH, uint32_t fl, int a,
                                               const float (&dj)[3]) {
    const bool oL = fl & f_open_lo(a), oH = fl & f_open_hi(a);
    const bool fL = fl & f_far_lo(a), fH = fl & f_far_hi(a);
    const float Cm1 = oL ? vm1 : Cc;
    const float Cp1 = oH ? vp1 : Cc;
    const float Cm2 = fL ? vm2 : Cm1;
    const float Cp2 = fH ? vp2 : Cp1;
    float DL, DH;
    if constexpr (BF) {
        const int bf = (fl & F_BF) ? 1 : 0;
        // face diffusivity by the biofilm count of its two voxels (0, 1,
        // 2); selected, not indexed, so the table stays in registers
        const int nl = bf + ((fl & f_nbf_lo(a)) ? 1 : 0);
        const int nh = bf + ((fl & f_nbf_hi(a)) ? 1 : 0);
        DL = oL ? (nl == 0 ? dj[0] : (nl == 1 ? dj[1] : dj[2])) : 0.f;
        DH = oH ? (nh == 0 ? dj[0] : (nh == 1 ? dj[1] : dj[2])) : 0.f;
    } else {
        DL = oL ? dj[0] : 0.f;
        DH = oH ? dj[0] : 0.f;
    }
    // out += D_hi (C+1 - C) + D_lo (C-1 - C)
    out = out + (DH * (Cp1 - Cc) + DL * (Cm1 - Cc));
    // upwind face values: the stencil is chosen first and limited once
    // (the same function of the same three values as choosing between
    // the two limited candidates)
    const bool rH = uH >= 0.f, rL = uL >= 0.f;
    const float fh = muscl(rH ? Cc : Cp1, rH ? Cm1 : Cp2, rH ? Cp1 : Cc);
    const float flo = muscl(rL ? Cm1 : Cc, rL ? Cm2 : Cp1, rL ? Cc : Cm1);
    // out -= u_hi f_hi - u_lo f_lo
    out = out - (uH * fh - uL * flo);
    divu = divu + (uH - uL);
}

// transport() of one chemical at one voxel (prtlb_3d.py:1182-1208), loading
// its neighbours and faces from global memory (the compacted-list kernels).
// INNER: the voxel is at least three planes from the inlet and two from
// every other face of the grid, so no neighbour position needs clamping and
// no neighbour lies on the inlet plane (no feed to substitute): the same
// values from fewer instructions.
// The face velocities of one voxel, low and high face of each of its ND axes
// (in Axes<ND> order).  They do not change during a run.
struct VoxelFaces {
    float lo[3], hi[3];
};

template <int ND>
__device__ __forceinline__ VoxelFaces load_faces(const Grid& g, const VoxelPos& v,
                                                 const float* const* __restrict__ face) {
    VoxelFaces fc;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
        const int a = Axes<ND>::ax(i);
        const int fi = face_lo(g, v, a);
        fc.lo[i] = ld_early(face[a] + fi);
        fc.hi[i] = ld_early(face[a] + fi + face_step(g, a));
    }
    return fc;
}

template <int ND, bool BF, bool INNER = false>
__device__ __forceinline__ float transport_one(const float* __restrict__ Cj, const Grid& g,
                                               const VoxelPos& v, uint32_t fl,
                                               const VoxelFaces& fc, float Cc,
                                               bool pin, float feed, const float (&dj)[3]) {
    float out = 0.f;
    float divu = 0.f;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
        const int a = Axes<ND>::ax(i);
        const int s = stride(g, a);
        float vm1, vp1, vm2, vp2;
        if constexpr (INNER) {
            vm1 = ld_early(Cj + (v.c - s));
            vp1 = ld_early(Cj + (v.c + s));
            vm2 = ld_early(Cj + (v.c - 2 * s));
            vp2 = ld_early(Cj + (v.c + 2 * s));
        } else {
            const int p = v.p[a];
            const int n = extent(g, a);
            // clamped (edge-replicated) neighbour positions
            const int pm1 = p > 0 ? p - 1 : 0, pm2 = p > 1 ? p - 2 : 0;
            const int pp1 = p < n - 1 ? p + 1 : n - 1, pp2 = p < n - 2 ? p + 2 : n - 1;
            const int x0 = v.p[0];
            const int xm1 = (a == 0) ? pm1 : x0, xm2 = (a == 0) ? pm2 : x0;
            const int xp1 = (a == 0) ? pp1 : x0, xp2 = (a == 0) ? pp2 : x0;
            // all four neighbours are loaded before the flags choose among
            // them (clamped addresses are always in the grid)
            vm1 = ld_c(Cj, v.c + (pm1 - p) * s, xm1, pin, feed);
            vp1 = ld_c(Cj, v.c + (pp1 - p) * s, xp1, pin, feed);
            vm2 = ld_c(Cj, v.c + (pm2 - p) * s, xm2, pin, feed);
            vp2 = ld_c(Cj, v.c + (pp2 - p) * s, xp2, pin, feed);
        }
        transport_axis<BF>(out, divu, Cc, vm1, vm2, vp1, vp2, fc.lo[i], fc.hi[i], fl, a, dj);
    }
    return out + Cc * divu;
}

// The reaction terms (rate_biotic, rate_abiotic, reaction: prtlb_3d.py:1224-1367)
// at one voxel, plus the reversible-sorption exchange (no reference counterpart).
template <int NS>
__device__ __forceinline__ void reaction(const float (&C)[NS], float surf,
                                         const prt_adr_params& p, float (&dC)[NS]) {
#pragma unroll
    for (int j = 0; j < NS; ++j) dC[j] = 0.f;
    float R = 0.f;
    if (p.biotic_on) {
        R = p.ks_donor_pos ? (p.k * C[0]) / (p.ks_donor + C[0]) : p.k * C[0];
        if (NS > 1) R = R * (p.ks_acceptor_pos ? C[NS > 1 ? 1 : 0] / (p.ks_acceptor + C[NS > 1 ? 1 : 0])
                                               : C[NS > 1 ? 1 : 0]);
        if (NS > 3 && p.coupled) R = (R * C[NS > 3 ? 3 : 0]) / p.c3_init;
        // caps: R <= 1/2 min(C0 / dt, C1 / (alpha dt))
        float lim = C[0] / p.dt;
        if (NS > 1 && p.alpha_cap) lim = np_min(lim, C[NS > 1 ? 1 : 0] / p.alpha_dt);
        R = np_min(R, 0.5f * lim);
    }
    float Ra = 0.f;
    if (p.abio_on) {
        float cj = 0.f;
#pragma unroll
        for (int j = 0; j < NS; ++j)
            if (j == p.j_ab) cj = C[j];
        Ra = p.surface_only ? (p.ka * cj) * surf : p.ka * cj;
        Ra = np_min(Ra, (0.5f * cj) / p.dt);
    }
    if (p.biotic_on) {
        dC[0] = -R;
        if (NS > 1) dC[NS > 1 ? 1 : 0] = p.neg_alpha * R;
        if (NS > 2) dC[NS > 2 ? 2 : 0] = p.prod_coef * R;
        if (NS > 3) dC[NS > 3 ? 3 : 0] = p.yield_ * R - p.kd * C[NS > 3 ? 3 : 0];
    } else {
        // R is the float32 scalar 0: -R, -alpha R, coef R are zeros, biomass 0
    }
    if (p.abio_on) {
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (j == p.j_ab) dC[j] = dC[j] - Ra;
        }
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (j == p.j_mk && p.j_mk != p.j_ab) dC[j] = dC[j] + Ra;
        }
    }
    if (p.sorp_on) {
        float c = 0.f, s = 0.f;
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (j == p.j_c) c = C[j];
            if (j == p.j_s) s = C[j];
        }
        float r = p.k_sorp * (c - s * p.inv_kd_sorp);
        r = np_min(r, (0.5f * c) / p.dt);
        r = np_max(r, -((0.5f * s) / p.dt));
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (j == p.j_c) dC[j] = dC[j] - r;
            if (j == p.j_s) dC[j] = dC[j] + r;
        }
    }
}

// The rest of step() at one solute voxel (prtlb_3d.py:1392-1413) once the
// transport terms T of the moving chemicals are known: the reaction terms
// (with the surface weight of a surface-only abiotic reaction), forward
// Euler and the clip at zero.  C holds the voxel's values after the inlet
// pin.
template <int ND, int NS>
__device__ __forceinline__ void adr_update(const float (&C)[NS], const float (&T)[NS], uint32_t fl,
                                           const prt_adr_params& p, float (&cn)[NS]) {
    float surf = 0.f;
    if (p.abio_on && p.surface_only) {
        float nface = 0.f;
#pragma unroll
        for (int i = 0; i < ND; ++i) {
            const int a = Axes<ND>::ax(i);
            nface = nface + ((fl & f_open_lo(a)) ? 0.f : 1.f);
            nface = nface + ((fl & f_open_hi(a)) ? 0.f : 1.f);
        }
        surf = nface / (float)(2 * ND);
    }
    float dC[NS];
    reaction<NS>(C, surf, p, dC);
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        const bool mv = (p.moving_mask >> j) & 1u;
        const float rhs = mv ? (T[j] + dC[j]) : dC[j];
        const float v = C[j] + p.dt * rhs;
        cn[j] = np_max(v, 0.f);
    }
}

// step() at one solute voxel (see adr_voxel), its flags and position known.
template <int ND, int NS, bool BF, bool INNER>
__device__ __forceinline__ void adr_voxel_body(const AdrDev& d, const prt_adr_params& p,
                                               long long n, int c, uint32_t fl,
                                               const VoxelPos& v, const VoxelFaces& fc) {
    const int N = (int)d.g.n;
    const float* __restrict__ Cin = d.buf[(n - 1) & 1];
    float* __restrict__ Cout = d.buf[n & 1];
    const bool x0 = fl & F_X0;
    float C[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        const bool pin = (p.pinned_mask >> j) & 1u;
        C[j] = (pin && x0) ? p.feed[j] : Cin[j * N + c];
    }
    float T[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        T[j] = 0.f;
        if ((p.moving_mask >> j) & 1u) {
            const bool pin = (p.pinned_mask >> j) & 1u;
            const float dj[3] = {p.dface[j][0], p.dface[j][1], p.dface[j][2]};
            T[j] = transport_one<ND, BF, INNER>(Cin + j * N, d.g, v, fl, fc, C[j], pin,
                                                p.feed[j], dj);
        }
    }
    float cn[NS];
    adr_update<ND, NS>(C, T, fl, p, cn);
    const int slot = d.slot_of_step[n];
    float* __restrict__ lad = slot >= 0 ? d.ladder + (long long)slot * NS * N : nullptr;
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        Cout[j * N + c] = cn[j];
        if (lad) lad[j * N + c] = cn[j];
    }
}

// What one transport step needs of solute voxel number kk (compacted C-order
// list) that does not change during a run: its voxel index, flags,
// position and face velocities.
struct VoxelSetup {
    int c;
    uint32_t fl;
    VoxelPos v;
    VoxelFaces fc;
};

template <int ND>
__device__ __forceinline__ VoxelSetup voxel_setup(const AdrDev& d, long long kk) {
    VoxelSetup s;
    s.c = d.idx[kk];
    s.fl = d.flags[s.c];
    s.v = voxel_pos(s.c, d.div_z, d.div_y);
    s.fc = load_faces<ND>(d.g, s.v, d.face);
    return s;
}

// One transport step of a solute voxel at step n: reads the state after
// step n-1 from buf[(n-1)&1], writes the state after step n to buf[n&1]
// and, when n is a snapshot step, to its ladder slot.  A warp whose voxels
// all lie inside the grid's interior (see transport_one) takes the interior
// form; the two forms give the same bits.
template <int ND, int NS, bool BF = true>
__device__ __forceinline__ void adr_voxel_step(const AdrDev& d, const prt_adr_params& p,
                                               long long n, const VoxelSetup& s) {
    const Grid& g = d.g;
    const VoxelPos& v = s.v;
    const bool inner = v.p[0] >= 3 && v.p[0] <= g.nx - 3 &&
                       (ND == 2 || (v.p[1] >= 2 && v.p[1] <= g.ny - 3)) && v.p[2] >= 2 &&
                       v.p[2] <= g.nz - 3;
    if (__all_sync(__activemask(), inner))
        adr_voxel_body<ND, NS, BF, true>(d, p, n, s.c, s.fl, v, s.fc);
    else
        adr_voxel_body<ND, NS, BF, false>(d, p, n, s.c, s.fl, v, s.fc);
}

// The same for solute voxel number kk (compacted C-order list).
template <int ND, int NS, bool BF = true>
__device__ __forceinline__ void adr_voxel(const AdrDev& d, const prt_adr_params& p, long long n,
                                          long long kk) {
    adr_voxel_step<ND, NS, BF>(d, p, n, voxel_setup<ND>(d, kk));
}

// The check of the time loop at step `end` (prtlb_3d.py:1499-1543), in
// float64 like the reference's arrays of Python floats: running scale,
// per-check change, geometric-tail remainder `rest`, the progress record,
// and the stop decision.
__device__ __forceinline__ double npd_max(double a, double b) { return (a >= b || a != a) ? a : b; }

__device__ inline void adr_check(AdrCtrl* ctrl, const float* __restrict__ means, long long end,
                                 ProgressRec* log, int log_cap) {
    const int ns = ctrl->ns;
    double cur[PRT_MAX_SPECIES], stepc[PRT_MAX_SPECIES];
    double change = 0.0, rest = 0.0;
    bool first = true;
    for (int j = 0; j < ns; ++j) {
        cur[j] = (double)means[j];
        ctrl->scale[j] = npd_max(ctrl->scale[j], fabs(cur[j]));
        stepc[j] = fabs(cur[j] - ctrl->prev[j]) / ctrl->scale[j];
        const double r = ctrl->prev_change[j] > 0 ? stepc[j] / ctrl->prev_change[j] : 0.0;
        double rj = (r < 1.0) ? stepc[j] * r / npd_max(1.0 - r, 1e-12) : INFINITY;
        if (!isfinite(rj)) rj = INFINITY;
        if (first) {
            change = stepc[j];
            rest = rj;
            first = false;
        } else {
            change = (change != change) ? change : ((stepc[j] != stepc[j]) ? stepc[j] : fmax(change, stepc[j]));
            rest = fmax(rest, rj);
        }
    }
    if (ctrl->nlog < log_cap) {
        ProgressRec& rec = log[ctrl->nlog];
        rec.n = end;
        rec.mean0 = cur[0];
        rec.value = isfinite(rest) ? rest : change;
    }
    ctrl->nlog += 1;
    ctrl->checks += 1;
    ctrl->last_rest = rest;
    if (ctrl->until_conv && end >= 10ll * ctrl->check && rest <= ctrl->tol) {
        ctrl->converged = 1;
        ctrl->done = 1;
    } else {
        for (int j = 0; j < ns; ++j) {
            ctrl->prev[j] = cur[j];
            ctrl->prev_change[j] = stepc[j];
        }
    }
}

// Sum of leaf `leaf` of numpy's float32 pairwise tree over the solute
// values s[idx[...]]: under 8 values sequentially from 0, otherwise eight
// interleaved accumulators ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)) and a tail.
__device__ inline float leaf_sum(const float* __restrict__ s, const int* __restrict__ idx,
                                 const PairTree& t, int leaf) {
    const int* ix = idx + t.leaf_start[leaf];
    const int len = t.leaf_len[leaf];
    float res;
    if (len < 8) {
        res = 0.f;
        for (int i = 0; i < len; ++i) res = res + s[ix[i]];
    } else {
        float r0 = s[ix[0]], r1 = s[ix[1]], r2 = s[ix[2]], r3 = s[ix[3]];
        float r4 = s[ix[4]], r5 = s[ix[5]], r6 = s[ix[6]], r7 = s[ix[7]];
        int i = 8;
        for (; i < len - (len % 8); i += 8) {
            r0 = r0 + s[ix[i + 0]];
            r1 = r1 + s[ix[i + 1]];
            r2 = r2 + s[ix[i + 2]];
            r3 = r3 + s[ix[i + 3]];
            r4 = r4 + s[ix[i + 4]];
            r5 = r5 + s[ix[i + 5]];
            r6 = r6 + s[ix[i + 6]];
            r7 = r7 + s[ix[i + 7]];
        }
        res = ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7));
        for (; i < len; ++i) res = res + s[ix[i]];
    }
    return res;
}

// The inner levels of the tree for one species (the whole block takes
// part), then mean = (0 + sum) / nm in float32 as ndarray.mean() does.
// L2: the node values are read through L2 (other blocks of the launch wrote
// the leaves).
template <bool L2 = false>
__device__ inline void tree_mean(const PairTree& t, long long nm, float* v, float* mean) {
    for (int h = 0; h < t.nlevel; ++h) {
        for (int i = t.level_off[h] + threadIdx.x; i < t.level_off[h + 1]; i += blockDim.x) {
            const float* a = v + t.inner_l[i];
            const float* b = v + t.inner_r[i];
            v[t.nleaf + i] = L2 ? __ldcg(a) + __ldcg(b) : *a + *b;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float sum = t.root >= 0 ? 0.f + v[t.root] : 0.f;
        *mean = sum / (float)nm;  // 0/0 -> NaN for an empty pore space, as numpy
    }
}

}  // namespace prt
