// adr.cu -- the transport step of PRT-LB (solve_adr, prtlb_3d.py:781-1595)
// for sm_100a: finite-volume advection (MUSCL/minmod), harmonic-mean
// diffusion, the C div(u) correction, the inlet Dirichlet feed, the reaction
// source terms, forward Euler and the clip, fused into one launch per step.
//
// This file is compiled with -fmad=false.  The reference integrates in
// float32 with numpy, one rounding per operation; with no fused multiply-add
// and the reference's operation order kept below, every voxel of every step
// is bit-identical to it, and so are the convergence means (numpy's float32
// pairwise summation is replayed by adr_means_*), the stop step and the
// snapshots.
#include "adr_core.cuh"

namespace prt {

// 128-thread blocks: at 64^3 (117 164 solute voxels, 148 SMs) the finer
// blocks balance the SMs better than 256 (5.30 -> 5.01 us per step; the
// same at 128^3; 64 threads 5.08 us).
constexpr int kAdrThreads = 128;

// One transport step n = n_base + kstep + 1 over every solute voxel (one
// thread each; rock voxels are never touched and stay 0 in every buffer).
// Launched with programmatic stream serialisation: what does not change
// during a run (the voxel's index, flags, position and face velocities) is
// read while the previous step drains; the control block and the
// concentrations only after griddepcontrol.wait.
// late: the next step is let in after this one's stores (see pdl_late).
template <int ND, int NS, bool BF>
__global__ void __launch_bounds__(kAdrThreads) adr_step_kernel(AdrDev d, prt_adr_params p,
                                                               const AdrCtrl* __restrict__ ctrl,
                                                               int kstep, int late) {
    if (!late) griddep_launch_dependents();
    const long long kk = (long long)blockIdx.x * kAdrThreads + threadIdx.x;
    const bool live = kk < d.nm;
    VoxelSetup s;
    if (live) s = voxel_setup<ND>(d, kk);
    griddep_wait();
    const long long n = ctrl->n_base + kstep + 1;
    if (ctrl->done || n > ctrl->limit) return;  // uniform over the grid
    if (!live) return;
    adr_voxel_step<ND, NS, BF>(d, p, n, s);
    if (late) griddep_launch_dependents();
}

// ---------------------------------------------------------------------------
// set-up (solve_adr 9.1-9.8, prtlb_3d.py:831-1158, 1425-1440)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool is_m(const uint8_t* mat, long long c, int pore, int bf) {
    const int v = mat[c];
    return v == pore || (bf >= 0 && v == bf);
}
__device__ __forceinline__ bool is_bf(const uint8_t* mat, long long c, int bf) {
    return bf >= 0 && mat[c] == bf;
}

__global__ void adr_flags_kernel(const uint8_t* __restrict__ mat, Grid g, int nd, int pore,
                                 int bfc, uint32_t* __restrict__ flags, uint8_t* __restrict__ mflag) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.n) return;
    const VoxelPos v = voxel_pos(c, g);
    const bool m = is_m(mat, c, pore, bfc);
    uint32_t fl = 0;
    if (m) fl |= F_M;
    if (is_bf(mat, c, bfc)) fl |= F_BF;
    if (m && v.p[0] == 0) fl |= F_X0;
    for (int i = 0; i < nd; ++i) {
        const int a = (nd == 3) ? i : (i == 0 ? 0 : 2);
        const int p = v.p[a];
        const int n = extent(g, a);
        const long long s = stride(g, a);
        const int pm1 = p > 0 ? p - 1 : 0, pm2 = p > 1 ? p - 2 : 0;
        const int pp1 = p < n - 1 ? p + 1 : n - 1, pp2 = p < n - 2 ? p + 2 : n - 1;
        const long long cm1 = c + (long long)(pm1 - p) * s, cm2 = c + (long long)(pm2 - p) * s;
        const long long cp1 = c + (long long)(pp1 - p) * s, cp2 = c + (long long)(pp2 - p) * s;
        const bool oL = m && is_m(mat, cm1, pore, bfc);
        const bool oH = m && is_m(mat, cp1, pore, bfc);
        const bool fL = oL && is_m(mat, cm2, pore, bfc);
        const bool fH = oH && is_m(mat, cp2, pore, bfc);
        if (oL) fl |= f_open_lo(a);
        if (oH) fl |= f_open_hi(a);
        if (fL) fl |= f_far_lo(a);
        if (fH) fl |= f_far_hi(a);
        if (is_bf(mat, cm1, bfc)) fl |= f_nbf_lo(a);
        if (is_bf(mat, cp1, bfc)) fl |= f_nbf_hi(a);
    }
    flags[c] = fl;
    mflag[c] = m ? 1 : 0;
}

// Face velocities u_f = 1/2 (u_lo + u_hi) on open faces, 0 on closed ones,
// from u = vel / u_scale (float32 division) masked to the solute voxels
// (prtlb_3d.py:860-865, 1092-1135).  Face f of axis a lies between voxels
// clamp(f-1) and clamp(f); faces 0 and n_a are the domain faces.
__global__ void adr_faces_kernel(const uint8_t* __restrict__ mat, const float* __restrict__ vcomp,
                                 Grid g, int a, int pore, int bfc, float u_scale,
                                 float* __restrict__ face) {
    const int fa = extent(g, a) + 1;
    const long long nf = g.n / extent(g, a) * fa;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nf) return;
    int q[3];
    const int dims[3] = {a == 0 ? fa : g.nx, a == 1 ? fa : g.ny, a == 2 ? fa : g.nz};
    unsigned long long r = (unsigned long long)t;
    q[2] = (int)(r % (unsigned)dims[2]);
    r /= (unsigned)dims[2];
    q[1] = (int)(r % (unsigned)dims[1]);
    q[0] = (int)(r / (unsigned)dims[1]);
    const int f = q[a];
    const int n = extent(g, a);
    const int plo = f - 1 < 0 ? 0 : f - 1;
    const int phi = f > n - 1 ? n - 1 : f;
    int ql[3] = {q[0], q[1], q[2]}, qh[3] = {q[0], q[1], q[2]};
    ql[a] = plo;
    qh[a] = phi;
    const long long cl = ((long long)ql[0] * g.ny + ql[1]) * g.nz + ql[2];
    const long long ch = ((long long)qh[0] * g.ny + qh[1]) * g.nz + qh[2];
    const bool ml = is_m(mat, cl, pore, bfc), mh = is_m(mat, ch, pore, bfc);
    float u = 0.f;
    if (ml && mh) {
        const float ul = vcomp[cl] / u_scale;
        const float uh = vcomp[ch] / u_scale;
        u = 0.5f * (ul + uh);
    }
    face[t] = u;
}

// Initial state (initial(), prtlb_3d.py:1425-1440) into buffer 0 and slot 0.
__global__ void adr_init_kernel(const uint32_t* __restrict__ flags, Grid g, prt_adr_params p,
                                float* __restrict__ buf0, float* __restrict__ slot0) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.n) return;
    const uint32_t fl = flags[c];
    for (int j = 0; j < p.ns; ++j) {
        float v = 0.f;
        if (p.init_mode[j] == 1 && (fl & F_M)) v = p.init_value[j];
        if (p.init_mode[j] == 2 && (fl & F_BF)) v = p.init_value[j];
        buf0[(long long)j * g.n + c] = v;
        if (slot0) slot0[(long long)j * g.n + c] = v;
    }
}

// Order-preserving compaction of the solute voxels (C order), in three passes.
constexpr int kScanBlock = 1024;
__global__ void count_kernel(const uint8_t* __restrict__ mflag, long long n, int* __restrict__ cnt) {
    const long long c = (long long)blockIdx.x * kScanBlock + threadIdx.x;
    int v = (c < n && mflag[c]) ? 1 : 0;
    v = __syncthreads_count(v);
    if (threadIdx.x == 0) cnt[blockIdx.x] = v;
}
__global__ void scan_counts_kernel(int* __restrict__ cnt, int nb, long long* __restrict__ total) {
    // one thread: the block counts are few (n / 1024)
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long acc = 0;
    for (int i = 0; i < nb; ++i) {
        const int v = cnt[i];
        cnt[i] = (int)acc;
        acc += v;
    }
    *total = acc;
}
__global__ void scatter_kernel(const uint8_t* __restrict__ mflag, long long n,
                               const int* __restrict__ off, int* __restrict__ idx) {
    __shared__ int warp_tot[kScanBlock / 32];
    const long long c = (long long)blockIdx.x * kScanBlock + threadIdx.x;
    const int v = (c < n && mflag[c]) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int before = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[w] = __popc(bal);
    __syncthreads();
    int base = 0;
    for (int i = 0; i < w; ++i) base += warp_tot[i];
    if (v) idx[off[blockIdx.x] + base + before] = (int)c;
}

// ---------------------------------------------------------------------------
// numpy float32 pairwise means (the stop rule's `C[j][m].mean()`), per
// species: leaf sums (leaf_sum) then the tree levels (tree_mean)
// ---------------------------------------------------------------------------
__global__ void means_leaf_kernel(const float* __restrict__ src, long long N,
                                  const int* __restrict__ idx, PairTree t, int ns,
                                  float* __restrict__ vals) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)t.nleaf * ns) return;
    const int leaf = (int)(tid % t.nleaf);
    const int j = (int)(tid / t.nleaf);
    vals[(long long)j * (t.nleaf + t.ninner) + leaf] = leaf_sum(src + (long long)j * N, idx, t, leaf);
}

__global__ void means_tree_kernel(PairTree t, long long nm, float* __restrict__ vals,
                                  float* __restrict__ means) {
    const int j = blockIdx.x;
    tree_mean(t, nm, vals + (long long)j * (t.nleaf + t.ninner), means + j);
}

__global__ void adr_stop_kernel(AdrCtrl* ctrl, const float* __restrict__ means, ProgressRec* log,
                                int log_cap, cudaGraphConditionalHandle h, int use_handle) {
    if (threadIdx.x != 0) return;
    if (ctrl->done) {
        if (use_handle) cudaGraphSetConditional(h, 0);
        return;
    }
    const long long base = ctrl->n_base;
    const long long end = min(base + (long long)ctrl->check, ctrl->limit);
    if (end > base && end % ctrl->check == 0) adr_check(ctrl, means, end, log, log_cap);
    ctrl->n_base = end;
    if (end >= ctrl->limit) ctrl->done = 1;
    const int go = (!ctrl->done && end < ctrl->n_pause) ? 1 : 0;
    if (use_handle) cudaGraphSetConditional(h, go);
}

__global__ void adr_means_pick_kernel(const AdrCtrl* ctrl, const float* buf0, const float* buf1,
                                      const float** out) {
    // chooses the buffer holding the state at the end of the current chunk
    const long long end = min(ctrl->n_base + (long long)ctrl->check, ctrl->limit);
    *out = (end & 1) ? buf1 : buf0;
}

// means over the buffer the device picked (graph body: pointer comes from device memory)
__global__ void means_leaf_indirect_kernel(const AdrCtrl* __restrict__ ctrl, const float* const* src_p,
                                           long long N, const int* __restrict__ idx, PairTree t,
                                           int ns, float* __restrict__ vals) {
    if (ctrl->done) return;
    const long long base = ctrl->n_base;
    const long long end = min(base + (long long)ctrl->check, ctrl->limit);
    if (!(end > base && end % ctrl->check == 0)) return;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)t.nleaf * ns) return;
    const int leaf = (int)(tid % t.nleaf);
    const int j = (int)(tid / t.nleaf);
    vals[(long long)j * (t.nleaf + t.ninner) + leaf] =
        leaf_sum(*src_p + (long long)j * N, idx, t, leaf);
}

__global__ void means_tree_cond_kernel(const AdrCtrl* __restrict__ ctrl, PairTree t, long long nm,
                                       float* __restrict__ vals, float* __restrict__ means) {
    if (ctrl->done) return;
    const long long base = ctrl->n_base;
    const long long end = min(base + (long long)ctrl->check, ctrl->limit);
    if (!(end > base && end % ctrl->check == 0)) return;
    const int j = blockIdx.x;
    tree_mean(t, nm, vals + (long long)j * (t.nleaf + t.ninner), means + j);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// Blocks of `kern` the device holds at once (128 threads each).
template <class K>
static long long resident_blocks(K kern) {
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kAdrThreads, 0) !=
            cudaSuccess ||
        cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (long long)per_sm * sms;
}

// Steps go out with programmatic stream serialisation.  One whose blocks
// exceed one resident wave lets the next step launch at its start (128^3:
// 16.2 -> 15.3 us per step, four chemicals 44.5 -> 40.5); one that fits in
// one wave only after its stores (pdl_late), because released at the start
// the next step's blocks, all resident early, slowed the running one (64^3:
// 4.32 -> 5.56 us) where released at the end they cut the step to 3.66 us.
// PRT_PDL=0 launches every step plainly.
template <int ND, int NS>
static cudaError_t step_t(const AdrDev& d, const prt_adr_params& p, AdrCtrl* ctrl, int k,
                          cudaStream_t s) {
    if (d.nm <= 0) return cudaSuccess;
    auto kern = d.has_bf ? adr_step_kernel<ND, NS, true> : adr_step_kernel<ND, NS, false>;
    const long long nb = (d.nm + kAdrThreads - 1) / kAdrThreads;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)nb);
    cfg.blockDim = dim3(kAdrThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    const int late = pdl_late(nb <= resident_blocks(kern)) ? 1 : 0;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, d, p, ctrl, k, late);
}

template <int ND>
static cudaError_t step_nd(const AdrDev& d, const prt_adr_params& p, AdrCtrl* ctrl, int k,
                           cudaStream_t s) {
    switch (d.ns) {
        case 1: return step_t<ND, 1>(d, p, ctrl, k, s);
        case 2: return step_t<ND, 2>(d, p, ctrl, k, s);
        case 3: return step_t<ND, 3>(d, p, ctrl, k, s);
        case 4: return step_t<ND, 4>(d, p, ctrl, k, s);
        case 5: return step_t<ND, 5>(d, p, ctrl, k, s);
        case 6: return step_t<ND, 6>(d, p, ctrl, k, s);
        case 7: return step_t<ND, 7>(d, p, ctrl, k, s);
        case 8: return step_t<ND, 8>(d, p, ctrl, k, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t adr_launch_step(const AdrDev& d, const prt_adr_params& p, AdrCtrl* ctrl, int kstep,
                            cudaStream_t s) {
    return d.nd == 3 ? step_nd<3>(d, p, ctrl, kstep, s) : step_nd<2>(d, p, ctrl, kstep, s);
}

// float32 speed sqrt((v0^2 + v1^2) [+ v2^2]) the way numpy forms it
__global__ void speed_kernel(const float* __restrict__ vel, Grid g, int nd,
                             float* __restrict__ sp) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.n) return;
    const float v0 = vel[c];
    const float v1 = vel[g.n + c];
    float s = v0 * v0 + v1 * v1;
    if (nd == 3) {
        const float v2 = vel[2 * g.n + c];
        s = s + v2 * v2;
    }
    sp[c] = sqrtf(s);
}

// max |vel[a]| over the solute voxels (order-free: max is exact)
__global__ void vmax_kernel(const float* __restrict__ vel, const int* __restrict__ idx, long long nm,
                            long long n, int nd, unsigned* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float m[3] = {0.f, 0.f, 0.f};
    if (t < nm) {
        const long long c = idx[t];
        for (int a = 0; a < nd; ++a) m[a] = fabsf(vel[(long long)a * n + c]);
    }
    for (int a = 0; a < 3; ++a) {
        float v = m[a];
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0 && v > 0.f) atomicMax(out + a, __float_as_uint(v));
    }
}

__global__ void count_bf_kernel(const uint32_t* __restrict__ flags, long long n,
                                unsigned long long* out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int v = (c < n && (flags[c] & F_BF)) ? 1 : 0;
    v = __syncthreads_count(v);
    if (threadIdx.x == 0 && v) atomicAdd(out, (unsigned long long)v);
}

cudaError_t adr_launch_flags(const uint8_t* mat, const Grid& g, int nd, int pore, int bfc,
                             uint32_t* flags, uint8_t* mflag, cudaStream_t s) {
    const unsigned nb = (unsigned)((g.n + 255) / 256);
    adr_flags_kernel<<<nb, 256, 0, s>>>(mat, g, nd, pore, bfc, flags, mflag);
    return cudaGetLastError();
}

// mean_axial, mean_speed (numpy float32 pairwise means over the solute
// voxels) into means[0..1]; max |v_a| bits into vmax_bits[0..2]; biofilm
// voxel count into *nbf.  tmp: n floats of scratch.
cudaError_t adr_launch_vel_stats(const float* vel, const AdrDev& d, float* tmp, float* means,
                                 unsigned* vmax_bits, unsigned long long* nbf, cudaStream_t s) {
    const Grid& g = d.g;
    const unsigned nb = (unsigned)((g.n + 255) / 256);
    cudaError_t e;
    for (int which = 0; which < 2; ++which) {
        const float* src = vel;
        if (which == 1) {
            speed_kernel<<<nb, 256, 0, s>>>(vel, g, d.nd, tmp);
            src = tmp;
        }
        if (d.tree.nleaf > 0) {
            means_leaf_kernel<<<(unsigned)((d.tree.nleaf + 255) / 256), 256, 0, s>>>(
                src, g.n, d.idx, d.tree, 1, d.tree_vals);
        }
        means_tree_kernel<<<1, 256, 0, s>>>(d.tree, d.nm, d.tree_vals, means + which);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (d.nm > 0)
        vmax_kernel<<<(unsigned)((d.nm + 255) / 256), 256, 0, s>>>(vel, d.idx, d.nm, g.n, d.nd,
                                                                  vmax_bits);
    count_bf_kernel<<<nb, 256, 0, s>>>(d.flags, g.n, nbf);
    return cudaGetLastError();
}

// Face velocities and the initial state; the flags are already built.
cudaError_t adr_launch_setup(const uint8_t* mat, const float* vel, const prt_adr_params& p,
                             const AdrDev& d, cudaStream_t s) {
    const Grid& g = d.g;
    const unsigned nb = (unsigned)((g.n + 255) / 256);
    cudaError_t e;
    for (int i = 0; i < d.nd; ++i) {
        const int a = (d.nd == 3) ? i : (i == 0 ? 0 : 2);
        const int ext = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
        const long long nf = g.n / ext * (ext + 1);
        // velocity component of storage axis a: 3D -> a; 2D -> x: 0, y (stored as z): 1
        const int comp = (d.nd == 3) ? a : (a == 0 ? 0 : 1);
        adr_faces_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(
            mat, vel + (long long)comp * g.n, g, a, p.pore_code, p.biofilm_code, p.u_scale,
            const_cast<float*>(d.face[a]));
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    adr_init_kernel<<<nb, 256, 0, s>>>(d.flags, g, p, d.buf[0], d.ladder);
    return cudaGetLastError();
}

cudaError_t adr_launch_compact(const uint8_t* mflag, long long n, int* cnt, long long* total,
                               int* idx, cudaStream_t s) {
    const int nb = (int)((n + kScanBlock - 1) / kScanBlock);
    count_kernel<<<nb, kScanBlock, 0, s>>>(mflag, n, cnt);
    scan_counts_kernel<<<1, 32, 0, s>>>(cnt, nb, total);
    if (idx) scatter_kernel<<<nb, kScanBlock, 0, s>>>(mflag, n, cnt, idx);
    return cudaGetLastError();
}

cudaError_t adr_launch_means(const AdrDev& d, AdrCtrl* ctrl, int slot, float* means_out,
                             cudaStream_t s) {
    // explicit means of ladder slot `slot` (slot >= 0), outside the time loop
    (void)ctrl;
    const float* src = d.ladder + (long long)slot * d.ns * d.g.n;
    if (d.tree.nleaf > 0) {
        const long long nt = (long long)d.tree.nleaf * d.ns;
        means_leaf_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(src, d.g.n, d.idx, d.tree, d.ns,
                                                                       d.tree_vals);
    }
    means_tree_kernel<<<d.ns, 256, 0, s>>>(d.tree, d.nm, d.tree_vals, means_out);
    return cudaGetLastError();
}

cudaError_t adr_launch_chunk_means(const AdrDev& d, AdrCtrl* ctrl, const float** src_slot,
                                   float* means_out, cudaStream_t s) {
    adr_means_pick_kernel<<<1, 1, 0, s>>>(ctrl, d.buf[0], d.buf[1], src_slot);
    if (d.tree.nleaf > 0) {
        const long long nt = (long long)d.tree.nleaf * d.ns;
        means_leaf_indirect_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(
            ctrl, src_slot, d.g.n, d.idx, d.tree, d.ns, d.tree_vals);
    }
    means_tree_cond_kernel<<<d.ns, 256, 0, s>>>(ctrl, d.tree, d.nm, d.tree_vals, means_out);
    return cudaGetLastError();
}

cudaError_t adr_launch_stop(const AdrDev& d, AdrCtrl* ctrl, const float* means,
                            cudaGraphConditionalHandle h, int use_handle, cudaStream_t s) {
    adr_stop_kernel<<<1, 32, 0, s>>>(ctrl, means, d.log, d.log_cap, h, use_handle);
    return cudaGetLastError();
}

}  // namespace prt
