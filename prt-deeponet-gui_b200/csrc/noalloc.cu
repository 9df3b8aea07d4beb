// noalloc.cu -- prt_flow_noalloc: the flow solve with no device allocation.
//
// Who needs it: callers that cannot call cudaMalloc -- code running inside a
// host framework that owns the whole device pool (and forbids foreign
// allocations), real-time loops that must never block on the allocator, and
// plug-in hosts that hand out device buffers for inputs and outputs but no
// allocator.  They pass the material grid and the velocity output as device
// pointers they already own, plus a stream; every other byte the solve needs
// (both population lattices, the neighbour masks, the per-block partial sums
// and the control block) lives in one file-scope __device__ array compiled
// into the library.
//
// Limits and sharing:
//   - The array is kNoAllocScratchBytes (48 MiB) on every GPU that loads the
//     library, held until the process exits.  A grid whose scratch would not
//     fit is refused with PRT_E_INVALID and a message giving both sizes; 64^3
//     D3Q19 with float32 populations fits.
//   - All calls on one device share the array and it keeps the last call's
//     contents; each call clears what must start at zero (the lattices, the
//     pore count) itself.  Calls whose work overlaps on the GPU (different
//     streams or threads at the same time) race on the array and give wrong
//     results: serialise them.
//   - Every call looks up the array's device address (cudaGetSymbolAddress)
//     on the calling thread's current device, in the CUDA context current
//     there, and runs the solve on that device.  Nothing is cached between
//     calls, so a device reset or another current context between calls is
//     seen by the next call.
//   - The call returns only after its work on the stream has finished, on
//     success and on every error after the first launch, so the caller may
//     free or reuse d_vel_out as soon as it returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "prt_internal.h"

using namespace prt;

namespace {

constexpr size_t kNoAllocScratchBytes = 48u << 20;

// The scratch itself.  In host code this name is only a stand-in for the
// device symbol; the kernels get the address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[kNoAllocScratchBytes];

// the message goes where prt_last_error(NULL) reads it
int fail(int code, const std::string& msg) {
    prt::set_noctx_error(msg.c_str());
    return code;
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

__global__ void noalloc_ctrl_kernel(FlowCtrl* ctrl, const long long* count, long long nit,
                                    double tol, int every) {
    // control block of a fresh solve; the pore count comes from the device
    ctrl->it_base = 0;
    ctrl->nit = nit;
    ctrl->iters = 0;
    ctrl->nfluid = (long long)*count;
    ctrl->tol = tol;
    ctrl->prev = 0.0;
    ctrl->change = INFINITY;
    ctrl->every = every;
    ctrl->done = nit == 0 ? 1 : 0;
    ctrl->has_prev = 0;
    ctrl->converged = 0;
    ctrl->nonfinite = 0;
    ctrl->pad = 0;
}

}  // namespace

#define NCK(expr)                                                                      \
    do {                                                                               \
        cudaError_t _e = (expr);                                                       \
        if (_e != cudaSuccess)                                                         \
            return fail(_e == cudaErrorMemoryAllocation ? PRT_E_OOM : PRT_E_CUDA,      \
                        std::string(#expr) + ": " + cudaGetErrorString(_e));           \
    } while (0)

namespace {

// The solve after the argument checks; `launched` is set once work may be
// queued on the stream.
int noalloc_solve(const uint8_t* d_mat, const prt_flow_params* p, float* d_vel_out,
                  prt_flow_info* info, cudaStream_t s, bool& launched) {
    Grid g;
    g.nx = p->dims[0];
    g.ny = p->nd == 3 ? p->dims[1] : 1;
    g.nz = p->nd == 3 ? p->dims[2] : p->dims[1];
    g.n = (long long)g.nx * g.ny * g.nz;
    if (g.n >= (1ll << 31) || coord_bits(g.nx) + coord_bits(g.ny) + coord_bits(g.nz) > 32)
        return fail(PRT_E_INVALID, "grid too large");
    const int Q = p->nd == 3 ? 19 : 9;
    const size_t es = p->precision == PRT_FP64 ? 8 : (p->precision == PRT_FP16 ? 2 : 4);
    // scratch layout, sized for the worst case (every voxel pore):
    // control | count | 5 reduced sums | block counts | partials | flags |
    // pore list | voxel -> slot map | 2 lattices
    const int nb_max = flow_blocks(g.n);
    const size_t o_ctrl = 0;
    const size_t o_count = o_ctrl + up256(sizeof(FlowCtrl));
    const size_t o_out5 = o_count + 256;
    const size_t o_cnt = o_out5 + 256;
    const size_t o_part = o_cnt + up256((size_t)((g.n + 1023) / 1024) * 4);
    const size_t o_flag = o_part + up256((size_t)nb_max * 5 * sizeof(double));
    const size_t o_cells = o_flag + up256((size_t)g.n);
    const size_t o_imap = o_cells + up256((size_t)g.n * 4);
    const size_t o_lat = o_imap + up256((size_t)g.n * 4);
    const size_t need = o_lat + (size_t)2 * Q * g.n * es;
    if (need > kNoAllocScratchBytes)
        return fail(PRT_E_INVALID,
                    "this grid needs " + std::to_string(need) + " bytes of scratch but the "
                    "allocation-free solve has " + std::to_string(kNoAllocScratchBytes) +
                    "; use prt_flow / prt_flow_dev");
    // the array's address in the context current on this thread's device
    void* base = nullptr;
    NCK(cudaGetSymbolAddress(&base, g_scratch));
    unsigned char* sb = static_cast<unsigned char*>(base);
    FlowCtrl* ctrl = reinterpret_cast<FlowCtrl*>(sb + o_ctrl);
    long long* count = reinterpret_cast<long long*>(sb + o_count);
    double* out5 = reinterpret_cast<double*>(sb + o_out5);
    int* cnt = reinterpret_cast<int*>(sb + o_cnt);
    double* parts = reinterpret_cast<double*>(sb + o_part);
    uint8_t* flag = sb + o_flag;
    int* cells = reinterpret_cast<int*>(sb + o_cells);
    int* imap = reinterpret_cast<int*>(sb + o_imap);
    void* f = sb + o_lat;

    float scale = 1.f;
    if (p->precision == PRT_FP16) {
        const double g0 = std::fabs(p->force) > 0 ? std::fabs(p->force) : 1e-6;
        scale = (float)std::ldexp(1.0, (int)std::floor(std::log2(1.0 / g0)));
    }
    LbParams k;
    fill_lbconst(k, p->nd, p->force, p->tau, p->magic, scale);

    // everything that must start at zero is cleared here: the array keeps
    // whatever the previous call left
    // pore-only layout: flags, count, pore list, voxel -> slot map
    launched = true;
    NCK(flow_launch_flags(d_mat, g.n, 2, flag, s));
    NCK(adr_launch_compact(flag, g.n, cnt, count, nullptr, s));
    long long nfluid = 0;
    NCK(cudaMemcpyAsync(&nfluid, count, sizeof(nfluid), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
    if ((long long)2 * Q * nfluid >= (1ll << 31))
        return fail(PRT_E_INVALID, "more pore voxels than the 32-bit lattice offsets hold");
    NCK(adr_launch_compact(flag, g.n, cnt, count, cells, s));
    NCK(cudaMemsetAsync(imap, 0xff, (size_t)g.n * 4, s));
    FlowMap fm;
    fm.ys = coord_bits(g.nz);
    fm.xs = fm.ys + coord_bits(g.ny);
    NCK(flow_launch_imap(cells, (int)nfluid, imap, g, fm.ys, fm.xs, s));
    fm.nf = (int)nfluid;
    fm.cells = cells;
    fm.imap = imap;
    fm.nbr = nullptr;
    const int nb = std::max(flow_blocks(nfluid), 1);
    NCK(cudaMemsetAsync(f, 0, (size_t)2 * Q * nfluid * es, s));
    NCK(cudaMemsetAsync(d_vel_out, 0, (size_t)3 * g.n * sizeof(float), s));
    NCK(cudaMemsetAsync(parts, 0, (size_t)nb * 5 * sizeof(double), s));
    noalloc_ctrl_kernel<<<1, 1, 0, s>>>(ctrl, count, p->nit, p->tol, p->every);
    NCK(cudaGetLastError());

    // the time loop, launched directly (no graph objects), chunk by chunk;
    // kernels after the stop are no-ops, so a few chunks go out per check
    const long long chunks = (p->nit + p->every - 1) / p->every;
    long long sent = 0;
    FlowCtrl hc;
    memset(&hc, 0, sizeof(hc));
    hc.done = p->nit == 0 ? 1 : 0;
    while (!hc.done && sent < chunks) {
        for (int r = 0; r < 8 && sent < chunks; ++r, ++sent) {
            for (int kk = 0; kk < p->every; ++kk)
                NCK(flow_launch_step(p->nd, p->precision, (kk & 1) != 0, kk == p->every - 1, f,
                                     fm, g, k, ctrl, kk, parts, s));
            NCK(flow_launch_check(ctrl, parts, nb, cudaGraphConditionalHandle(0), 0, s));
        }
        NCK(cudaMemcpyAsync(&hc, ctrl, sizeof(hc), cudaMemcpyDeviceToHost, s));
        NCK(cudaStreamSynchronize(s));
    }
    NCK(cudaMemcpyAsync(&hc, ctrl, sizeof(hc), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
    NCK(flow_launch_moments(p->nd, p->precision, (hc.iters & 1) != 0, f, fm, g, k, d_vel_out,
                            parts, s));
    NCK(flow_launch_final_reduce(parts, nb, out5, s));
    double o5[5];
    NCK(cudaMemcpyAsync(o5, out5, sizeof(o5), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
    if (info) {
        memset(info, 0, sizeof(*info));
        info->iters = hc.iters;
        info->converged = hc.converged;
        info->change = hc.change;
        info->fluid_cells = (int64_t)nfluid;
        info->ux_sum = o5[0];
        info->mass = o5[1];
        info->speed_sum = o5[2];
        info->umax = o5[3];
        info->nonfinite = (int64_t)llround(o5[4]);
        const double nu = (p->tau - 0.5) / 3.0;
        info->permeability = p->force != 0 ? nu * (o5[0] / (double)g.n) / p->force : 0.0;
        info->fp16_scale = scale;
    }
    return PRT_OK;
}

}  // namespace

extern "C" int prt_flow_noalloc(const uint8_t* d_mat, const prt_flow_params* p, float* d_vel_out,
                                prt_flow_info* info, void* stream) {
    prt::set_noctx_error("");  // a success leaves no earlier message behind
    if (!p || !d_mat || !d_vel_out) return fail(PRT_E_INVALID, "null argument");
    if (p->nd != 2 && p->nd != 3) return fail(PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < p->nd; ++i)
        if (p->dims[i] <= 0) return fail(PRT_E_INVALID, "grid dimensions must be positive");
    if (!(p->tau > 0.5))
        return fail(PRT_E_INVALID, "tau must exceed 0.5; the viscosity (tau-1/2)/3 is negative "
                                   "below it and the solver cannot run.");
    if (p->every <= 0 || (p->every & 1))
        return fail(PRT_E_INVALID, "the convergence interval must be a positive even number");
    if (p->precision < PRT_FP64 || p->precision > PRT_FP32_F32)
        return fail(PRT_E_INVALID, "unknown precision");
    if (p->nit < 0) return fail(PRT_E_INVALID, "negative iteration cap");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bool launched = false;
    const int rc = noalloc_solve(d_mat, p, d_vel_out, info, s, launched);
    // a failure after the first launch still waits for what was queued, so
    // no kernel of this call writes d_vel_out or the array after the return
    if (rc != PRT_OK && launched) cudaStreamSynchronize(s);
    return rc;
}
