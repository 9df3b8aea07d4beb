// physics.cu -- the statistics check_physics judges a transport result by
// (prtlb_3d.py:1632-1843), reduced on the device from the snapshots
// out (n_t, ns, voxels) float32 and the material grid.
//
// The rules and their messages stay on the host (prtlb_gpu.physics); the
// device supplies what they read:
//   non-finite counts over the whole result;
//   per chemical, the largest and smallest value over the pore voxels of
//   every snapshot and the largest |value| over the pore of the last one;
//   per snapshot, the largest donor value on the planes x = nx / 2 and
//   x = nx - 1 (every voxel of the plane);
//   on the last donor snapshot, the pore triples along x and how many of
//   them have neighbour differences of opposite sign (the checkerboard);
//   for each chemical j >= 1 against the donor, over the pore of every
//   snapshot: the means, the centred second moments and, given a scale s,
//   the largest |a_j - s a_0| (float32, as numpy forms it).
// Extremes and counts are exact whatever the order; the moments are float64
// sums (the host rules compare them with margins of 1e-4 and more).
#include "runtime_internal.h"

namespace prt {

namespace {

constexpr int kPhysThreads = 256;

// float -> unsigned key with the same order (NaN never reaches it)
__device__ __forceinline__ unsigned fkey(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

struct PhysGrid {
    long long n;  // voxels
    int nt, ns;
    FastDiv dyz;  // by ny * nz: the x of a voxel
    int nx;
};

// keys: [0, ns) max, [ns, 2 ns) min (as ~key, so atomicMax finds it),
// [2 ns, 3 ns) final |max|, [3 ns, 3 ns + nt) mid-plane max,
// [3 ns + nt, 3 ns + 2 nt) outlet-plane max; cnt: nan, inf.
// Each block gathers its extremes in shared memory and adds them to the
// global keys once, so the global atomics are one per key per block.
__global__ void __launch_bounds__(kPhysThreads)
    phys_extremes_kernel(const float* __restrict__ out, const uint8_t* __restrict__ mat, int pore,
                         PhysGrid p, unsigned* __restrict__ keys,
                         unsigned long long* __restrict__ cnt) {
    __shared__ unsigned sk[3 * PRT_MAX_SPECIES + 2 * PRT_PHYS_MAX_SNAPSHOTS];
    const int nkeys = 3 * p.ns + 2 * p.nt;
    for (int i = threadIdx.x; i < nkeys; i += kPhysThreads) sk[i] = 0;
    __syncthreads();
    const long long total = (long long)p.nt * p.ns * p.n;
    unsigned long long nnan = 0, ninf = 0;
    for (long long e = (long long)blockIdx.x * kPhysThreads + threadIdx.x; e < total;
         e += (long long)gridDim.x * kPhysThreads) {
        const float v = out[e];
        const long long c = e % p.n;
        const long long tj = e / p.n;
        const int j = (int)(tj % p.ns);
        const int t = (int)(tj / p.ns);
        if (v != v) {
            ++nnan;
            continue;
        }
        if (isinf(v)) ++ninf;
        if (mat[c] == pore) {
            atomicMax(sk + j, fkey(v));
            atomicMax(sk + p.ns + j, ~fkey(v));
            if (t == p.nt - 1) atomicMax(sk + 2 * p.ns + j, fkey(fabsf(v)));
        }
        if (j == 0) {
            const int x = (int)fast_div((unsigned)c, p.dyz);
            if (x == p.nx / 2) atomicMax(sk + 3 * p.ns + t, fkey(v));
            if (x == p.nx - 1) atomicMax(sk + 3 * p.ns + p.nt + t, fkey(v));
        }
    }
    if (nnan) atomicAdd(cnt, nnan);
    if (ninf) atomicAdd(cnt + 1, ninf);
    __syncthreads();
    for (int i = threadIdx.x; i < nkeys; i += kPhysThreads)
        if (sk[i]) atomicMax(keys + i, sk[i]);
}

// Pore triples along x of the last donor snapshot and the ones whose two
// neighbour differences have opposite signs: cnt[2], cnt[3].
__global__ void __launch_bounds__(kPhysThreads)
    phys_checker_kernel(const float* __restrict__ f, const uint8_t* __restrict__ mat, int pore,
                        PhysGrid p, unsigned long long* __restrict__ cnt) {
    const long long sx = p.n / p.nx;
    int trip = 0, flip = 0;
    const long long c = (long long)blockIdx.x * kPhysThreads + threadIdx.x;
    if (c < p.n) {
        const int x = (int)fast_div((unsigned)c, p.dyz);
        if (x >= 1 && x <= p.nx - 2 && mat[c - sx] == pore && mat[c] == pore &&
            mat[c + sx] == pore) {
            trip = 1;
            const float lo = f[c] - f[c - sx];
            const float hi = f[c + sx] - f[c];
            flip = (lo > 0.f && hi < 0.f) || (lo < 0.f && hi > 0.f);
        }
    }
    const int nt = __syncthreads_count(trip);
    const int nf = __syncthreads_count(flip);
    if (threadIdx.x == 0) {
        if (nt) atomicAdd(cnt + 2, (unsigned long long)nt);
        if (nf) atomicAdd(cnt + 3, (unsigned long long)nf);
    }
}

// Moments of the donor against chemical j over the pore of every snapshot.
// stage 0: sums[0] += a0, sums[1] += aj, sums[5] += 1;
// stage 1: sums[2] += (a0 - m0)^2, sums[3] += (aj - mj)^2,
//          sums[4] += (a0 - m0)(aj - mj) with m = sums / count;
// stage 2: keys[0] max of fkey(|aj - scale a0|) in float32.
__global__ void __launch_bounds__(kPhysThreads)
    phys_moment_kernel(const float* __restrict__ out, const uint8_t* __restrict__ mat, int pore,
                       PhysGrid p, int j, int stage, float scale, double* __restrict__ sums,
                       unsigned* __restrict__ key) {
    __shared__ double sh[3][kPhysThreads / 32];
    const long long total = (long long)p.nt * p.n;
    double m0 = 0.0, mj = 0.0;
    if (stage == 1 && sums[5] > 0) {
        m0 = sums[0] / sums[5];
        mj = sums[1] / sums[5];
    }
    double acc[3] = {0.0, 0.0, 0.0};
    unsigned kmax = 0;
    for (long long e = (long long)blockIdx.x * kPhysThreads + threadIdx.x; e < total;
         e += (long long)gridDim.x * kPhysThreads) {
        const long long c = e % p.n;
        if (mat[c] != pore) continue;
        const long long t = e / p.n;
        const float a0 = out[(t * p.ns) * p.n + c];
        const float aj = out[(t * p.ns + j) * p.n + c];
        if (stage == 0) {
            acc[0] += a0;
            acc[1] += aj;
            acc[2] += 1.0;
        } else if (stage == 1) {
            const double d0 = a0 - m0, dj = aj - mj;
            acc[0] += d0 * d0;
            acc[1] += dj * dj;
            acc[2] += d0 * dj;
        } else {
            const float dev = fabsf(__fsub_rn(aj, __fmul_rn(scale, a0)));
            kmax = max(kmax, fkey(dev));
        }
    }
    if (stage == 2) {
        if (kmax) atomicMax(key, kmax);
        return;
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int w = 0; w < kPhysThreads / 32; ++w) v += sh[threadIdx.x][w];
        const int slot = stage == 0 ? (threadIdx.x == 2 ? 5 : threadIdx.x) : 2 + threadIdx.x;
        atomicAdd(sums + slot, v);
    }
}

}  // namespace

}  // namespace prt

using namespace prt;

namespace {

float unkey(unsigned k) {
    const unsigned b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

}  // namespace


// d_out / d_mat may be NULL: the arrays staged by prt_physics_stage.
static int resolve(prt_ctx* ctx, const float*& d_out, const uint8_t*& d_mat, long long n,
                   long long nfloat) {
    PrepState& P = ctx->prep;
    if (!d_out) {
        if (P.staged_out != nfloat)
            return fail(ctx, PRT_E_STATE, "no staged result of this size (prt_physics_stage)");
        d_out = P.out.as<float>();
    }
    if (!d_mat) {
        if (P.staged_mat != n)
            return fail(ctx, PRT_E_STATE, "no staged material grid of this size (prt_physics_stage)");
        d_mat = P.mat.as<uint8_t>();
    }
    return PRT_OK;
}

extern "C" int prt_physics_stage(prt_ctx* ctx, const float* out, const uint8_t* mat, int32_t nd,
                                 const int32_t* dims, int32_t n_t, int32_t ns) {
    if (!ctx || !out || !mat || !dims) return fail(ctx, PRT_E_INVALID, "null argument");
    if (nd != 2 && nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < nd; ++i)
        if (dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    if (n_t < 1 || ns < 1) return fail(ctx, PRT_E_INVALID, "empty result");
    const Grid g = make_grid(nd, dims);
    CK(cudaSetDevice(ctx->device));
    PrepState& P = ctx->prep;
    const long long nf = (long long)n_t * ns * g.n;
    CK(P.out.ensure((size_t)nf * 4));
    CK(P.mat.ensure((size_t)g.n));
    CK(cudaMemcpyAsync(P.out.p, out, (size_t)nf * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(P.mat.p, mat, (size_t)g.n, cudaMemcpyHostToDevice, ctx->stream));
    P.staged_out = nf;
    P.staged_mat = g.n;
    return PRT_OK;
}

extern "C" int prt_physics_stats_dev(prt_ctx* ctx, const float* d_out, const uint8_t* d_mat,
                                     int32_t nd, const int32_t* dims, int32_t n_t, int32_t ns,
                                     int32_t pore_code, prt_physics_stats* st) {
    if (!ctx || !dims || !st) return fail(ctx, PRT_E_INVALID, "null argument");
    if (nd != 2 && nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < nd; ++i)
        if (dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    if (n_t < 1 || n_t > PRT_PHYS_MAX_SNAPSHOTS || ns < 1 || ns > PRT_MAX_SPECIES)
        return fail(ctx, PRT_E_INVALID, "between 1 and 256 snapshots of 1 to 8 chemicals");
    const Grid g = make_grid(nd, dims);
    if (g.n >= (1ll << 31)) return fail(ctx, PRT_E_INVALID, "grids of 2^31 voxels or more");
    int rc = resolve(ctx, d_out, d_mat, g.n, (long long)n_t * ns * g.n);
    if (rc != PRT_OK) return rc;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    PrepState& P = ctx->prep;
    const int nkeys = 3 * ns + 2 * n_t;
    CK(P.keys.ensure((size_t)(nkeys + 1) * sizeof(unsigned)));
    CK(P.sums.ensure(8 * sizeof(double) + 4 * sizeof(unsigned long long)));
    unsigned* keys = P.keys.as<unsigned>();
    double* sums = P.sums.as<double>();
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(sums + 8);
    CK(cudaMemsetAsync(keys, 0, (size_t)(nkeys + 1) * sizeof(unsigned), s));
    CK(cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned long long), s));
    PhysGrid p;
    p.n = g.n;
    p.nt = n_t;
    p.ns = ns;
    p.nx = g.nx;
    p.dyz = make_fastdiv((unsigned)(g.ny * g.nz));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    const int grid = nsm * 8;
    phys_extremes_kernel<<<grid, kPhysThreads, 0, s>>>(d_out, d_mat, pore_code, p, keys, cnt);
    CK(cudaGetLastError());
    const float* last0 = d_out + (long long)(n_t - 1) * ns * g.n;
    phys_checker_kernel<<<(unsigned)((g.n + kPhysThreads - 1) / kPhysThreads), kPhysThreads, 0, s>>>(
        last0, d_mat, pore_code, p, cnt);
    CK(cudaGetLastError());
    ctx->launches += 2;
    std::vector<unsigned> hk(nkeys);
    unsigned long long hc[4];
    CK(cudaMemcpyAsync(hk.data(), keys, (size_t)nkeys * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::memset(st, 0, sizeof(*st));
    st->n_nan = (int64_t)hc[0];
    st->n_inf = (int64_t)hc[1];
    st->n_triples = (int64_t)hc[2];
    st->n_flips = (int64_t)hc[3];
    // a key of 0 means no value was seen (no pore, or all of it NaN)
    for (int j = 0; j < ns; ++j) {
        st->has_pore[j] = hk[j] != 0;
        st->pore_max[j] = hk[j] ? unkey(hk[j]) : 0.f;
        st->pore_min[j] = hk[ns + j] ? unkey(~hk[ns + j]) : 0.f;
        st->final_absmax[j] = hk[2 * ns + j] ? unkey(hk[2 * ns + j]) : 0.f;
    }
    for (int t = 0; t < n_t; ++t) {
        st->mid_max[t] = unkey(hk[3 * ns + t]);
        st->end_max[t] = unkey(hk[3 * ns + n_t + t]);
    }
    return PRT_OK;
}

extern "C" int prt_physics_moments_dev(prt_ctx* ctx, const float* d_out, const uint8_t* d_mat,
                                       int32_t nd, const int32_t* dims, int32_t n_t, int32_t ns,
                                       int32_t pore_code, int32_t j, double* moments6) {
    if (!ctx || !dims || !moments6) return fail(ctx, PRT_E_INVALID, "null argument");
    if (nd != 2 && nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < nd; ++i)
        if (dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    if (n_t < 1 || ns < 2 || ns > PRT_MAX_SPECIES || j < 1 || j >= ns)
        return fail(ctx, PRT_E_INVALID, "chemical j must be 1 .. ns-1");
    const Grid g = make_grid(nd, dims);
    if (g.n >= (1ll << 31)) return fail(ctx, PRT_E_INVALID, "grids of 2^31 voxels or more");
    int rc = resolve(ctx, d_out, d_mat, g.n, (long long)n_t * ns * g.n);
    if (rc != PRT_OK) return rc;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    PrepState& P = ctx->prep;
    CK(P.sums.ensure(8 * sizeof(double) + 4 * sizeof(unsigned long long)));
    double* sums = P.sums.as<double>();
    CK(cudaMemsetAsync(sums, 0, 8 * sizeof(double), s));
    PhysGrid p;
    p.n = g.n;
    p.nt = n_t;
    p.ns = ns;
    p.nx = g.nx;
    p.dyz = make_fastdiv((unsigned)(g.ny * g.nz));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    const int grid = nsm * 8;
    for (int stage = 0; stage < 2; ++stage)
        phys_moment_kernel<<<grid, kPhysThreads, 0, s>>>(d_out, d_mat, pore_code, p, j, stage, 0.f,
                                                          sums, nullptr);
    CK(cudaGetLastError());
    ctx->launches += 2;
    double h[6];
    CK(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // count, mean0, meanj, var0, varj, cov (population)
    const double n = h[5];
    moments6[0] = n;
    moments6[1] = n > 0 ? h[0] / n : 0.0;
    moments6[2] = n > 0 ? h[1] / n : 0.0;
    moments6[3] = n > 0 ? h[2] / n : 0.0;
    moments6[4] = n > 0 ? h[3] / n : 0.0;
    moments6[5] = n > 0 ? h[4] / n : 0.0;
    return PRT_OK;
}

extern "C" int prt_physics_maxdev_dev(prt_ctx* ctx, const float* d_out, const uint8_t* d_mat,
                                      int32_t nd, const int32_t* dims, int32_t n_t, int32_t ns,
                                      int32_t pore_code, int32_t j, float scale, float* maxdev) {
    if (!ctx || !dims || !maxdev) return fail(ctx, PRT_E_INVALID, "null argument");
    if (nd != 2 && nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < nd; ++i)
        if (dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    if (n_t < 1 || ns < 2 || ns > PRT_MAX_SPECIES || j < 1 || j >= ns)
        return fail(ctx, PRT_E_INVALID, "chemical j must be 1 .. ns-1");
    const Grid g = make_grid(nd, dims);
    if (g.n >= (1ll << 31)) return fail(ctx, PRT_E_INVALID, "grids of 2^31 voxels or more");
    int rc = resolve(ctx, d_out, d_mat, g.n, (long long)n_t * ns * g.n);
    if (rc != PRT_OK) return rc;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    PrepState& P = ctx->prep;
    CK(P.keys.ensure(sizeof(unsigned)));
    unsigned* key = P.keys.as<unsigned>();
    CK(cudaMemsetAsync(key, 0, sizeof(unsigned), s));
    PhysGrid p;
    p.n = g.n;
    p.nt = n_t;
    p.ns = ns;
    p.nx = g.nx;
    p.dyz = make_fastdiv((unsigned)(g.ny * g.nz));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    phys_moment_kernel<<<nsm * 8, kPhysThreads, 0, s>>>(d_out, d_mat, pore_code, p, j, 2, scale,
                                                         nullptr, key);
    CK(cudaGetLastError());
    ctx->launches += 1;
    unsigned hk = 0;
    CK(cudaMemcpyAsync(&hk, key, sizeof(hk), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *maxdev = hk ? unkey(hk) : 0.f;
    return PRT_OK;
}
