// runtime.cu -- the C ABI of libprtlb.so (include/prtlb.h): contexts, device
// buffers, and the two time loops run as CUDA graphs with a device-side
// while-condition, so a whole flow solve or transport solve is one graph
// launch and the host waits once.
#include <cstdlib>
#include <new>

#include "runtime_internal.h"

using namespace prt;

namespace {
thread_local std::string g_create_error;
}  // namespace

// ===========================================================================
// context
// ===========================================================================
extern "C" int prt_abi_version(void) { return PRT_ABI_VERSION; }

extern "C" int prt_create(int device, prt_ctx** out) {
    if (!out) return PRT_E_INVALID;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        g_create_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return PRT_E_NODEV;
    }
    if (device < 0 || device >= n) {
        g_create_error = "device index out of range";
        return PRT_E_INVALID;
    }
    prt_ctx* c = new (std::nothrow) prt_ctx();
    if (!c) return PRT_E_OOM;
    c->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
    int l2 = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device);
    c->l2_bytes = l2;
    if (e != cudaSuccess) {
        g_create_error = std::string("cuda init failed: ") + cudaGetErrorString(e);
        delete c;
        return PRT_E_CUDA;
    }
    *out = c;
    return PRT_OK;
}

extern "C" void prt_destroy(prt_ctx* c) {
    if (!c) return;
    batch_detach(c);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->adr.release();
    c->prep.release();
    FlowState& f = c->flow;
    DevBuf* all[] = {&f.f,    &f.fluid, &f.partials, &f.ctrl, &f.out5, &f.count,
                     &f.mat,  &f.vel,   &f.flag,     &f.cnt,  &f.cells, &f.nbr};
    for (DevBuf* b : all) b->release();
    f.graph.release();
    for (int i = 0; i < 4; ++i)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" const char* prt_last_error(const prt_ctx* c) {
    return c ? c->err.c_str() : g_create_error.c_str();
}

// Message of a failed call that has no context (prt_flow_noalloc).
void prt::set_noctx_error(const char* msg) { g_create_error = msg ? msg : ""; }

extern "C" int64_t prt_kernel_launches(const prt_ctx* c) { return c ? c->launches : 0; }

extern "C" void* prt_stream(const prt_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int prt_last_timing(const prt_ctx* c, double* out4) {
    if (!c || !out4) return PRT_E_INVALID;
    for (int i = 0; i < 4; ++i) out4[i] = c->timing[i];
    return PRT_OK;
}

extern "C" size_t prt_sizeof(int which) {
    switch (which) {
        case 0: return sizeof(prt_flow_params);
        case 1: return sizeof(prt_flow_info);
        case 2: return sizeof(prt_adr_params);
        case 3: return sizeof(prt_adr_run_params);
        case 4: return sizeof(prt_adr_result);
        case 5: return sizeof(prt_adr_geom);
        case 6: return sizeof(prt_adr_stats);
        case 7: return sizeof(prt_physics_stats);
        default: return 0;
    }
}

// ===========================================================================
// flow
// ===========================================================================
// The upstream-slot table: by the working set against the L2 cache
// (flow_use_nbr), or always / never with PRT_NBR_TABLE=1 / 0.  Both ways
// give the same slots, so the fields are bit-identical either way.
static bool nbr_table_wanted(int q, long long nf, long long es, long long l2_bytes) {
    if (nf <= 0) return false;
    const char* v = std::getenv("PRT_NBR_TABLE");
    if (v && v[0] == '1') return true;
    if (v && v[0] == '0') return false;
    return flow_use_nbr(q, nf, es, l2_bytes);
}

// Flow solve in three parts, so the batched engine can run many set-up
// solves through one time loop: set-up (buffers, pore-only layout, control
// block, constants), the time loop, and the final field with its reductions.
int prt::flow_setup(prt_ctx* ctx, const uint8_t* d_mat, const prt_flow_params* p, float* d_vel) {
    if (!ctx || !p || !d_mat || !d_vel) return fail(ctx, PRT_E_INVALID, "null argument");
    if (p->nd != 2 && p->nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < p->nd; ++i)
        if (p->dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    if (!(p->tau > 0.5))
        return fail(ctx, PRT_E_INVALID,
                    "tau must exceed 0.5; the viscosity (tau-1/2)/3 is negative below it and the "
                    "solver cannot run.");
    if (p->every <= 0 || (p->every & 1))
        return fail(ctx, PRT_E_INVALID, "the convergence interval must be a positive even number");
    if (p->precision < PRT_FP64 || p->precision > PRT_FP32_F32)
        return fail(ctx, PRT_E_INVALID, "unknown precision");
    if (p->nit < 0) return fail(ctx, PRT_E_INVALID, "negative iteration cap");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    FlowState& F = ctx->flow;
    const Grid g = make_grid(p->nd, p->dims);
    const int Q = p->nd == 3 ? 19 : 9;
    const size_t es = p->precision == PRT_FP64 ? 8 : (p->precision == PRT_FP16 ? 2 : 4);
    if (g.n >= (1ll << 31) || coord_bits(g.nx) + coord_bits(g.ny) + coord_bits(g.nz) > 32)
        return fail(ctx, PRT_E_INVALID,
                    "grids of 2^31 voxels or more (or whose packed coordinates exceed 32 bits) "
                    "are not supported");
    // pore-only layout: flags, compacted voxel list, voxel -> slot map
    CK(F.flag.ensure((size_t)g.n));
    CK(F.cnt.ensure((size_t)((g.n + 1023) / 1024) * 4));
    CK(F.count.ensure(sizeof(long long)));
    CK(flow_launch_flags(d_mat, g.n, 2, F.flag.as<uint8_t>(), s));
    CK(adr_launch_compact(F.flag.as<uint8_t>(), g.n, F.cnt.as<int>(), F.count.as<long long>(),
                          nullptr, s));
    long long nfluid = 0;
    CK(cudaMemcpyAsync(&nfluid, F.count.p, sizeof(nfluid), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(F.cells.ensure((size_t)std::max(nfluid, 1ll) * 4));
    CK(F.fluid.ensure((size_t)g.n * 4));  // imap
    CK(adr_launch_compact(F.flag.as<uint8_t>(), g.n, F.cnt.as<int>(), F.count.as<long long>(),
                          F.cells.as<int>(), s));
    CK(cudaMemsetAsync(F.fluid.p, 0xff, (size_t)g.n * 4, s));
    F.fm.ys = coord_bits(g.nz);
    F.fm.xs = F.fm.ys + coord_bits(g.ny);
    CK(flow_launch_imap(F.cells.as<int>(), (int)nfluid, F.fluid.as<int>(), g, F.fm.ys, F.fm.xs,
                        s));
    ctx->launches += 7;
    if ((long long)2 * Q * nfluid >= (1ll << 31))
        return fail(ctx, PRT_E_INVALID,
                    "more pore voxels than the 32-bit lattice offsets hold (2 Q nf >= 2^31)");
    F.fm.nf = (int)nfluid;
    F.fm.cells = F.cells.as<int>();
    F.fm.imap = F.fluid.as<int>();
    F.fm.nbr = nullptr;
    if (nbr_table_wanted(Q, nfluid, (long long)es, ctx->l2_bytes)) {
        CK(F.nbr.ensure((size_t)flow_nbr_bytes(Q, nfluid)));
        CK(flow_launch_nbr(p->nd, F.fm, g, F.nbr.as<int>(), s));
        ctx->launches += 1;
        F.fm.nbr = F.nbr.as<int>();
    }
    F.nb = std::max(flow_blocks(nfluid), 1);
    CK(F.f.ensure((size_t)2 * Q * std::max(nfluid, 1ll) * es));  // two lattices
    CK(F.partials.ensure((size_t)F.nb * 5 * sizeof(double)));
    CK(F.ctrl.ensure(sizeof(FlowCtrl)));
    CK(F.out5.ensure(8 * sizeof(double)));

    // f = w_i everywhere, in both lattices: shifted storage h = 0; rock
    // voxels of the output velocity are 0
    CK(cudaMemsetAsync(F.f.p, 0, (size_t)2 * Q * nfluid * es, s));
    CK(cudaMemsetAsync(d_vel, 0, (size_t)3 * g.n * sizeof(float), s));
    CK(cudaMemsetAsync(F.partials.p, 0, (size_t)F.nb * 5 * sizeof(double), s));
    FlowCtrl hc{};
    hc.it_base = 0;
    hc.nit = p->nit;
    hc.iters = 0;
    hc.nfluid = (long long)nfluid;
    hc.tol = p->tol;
    hc.prev = 0;
    hc.change = INFINITY;
    hc.every = p->every;
    hc.done = p->nit == 0 ? 1 : 0;
    CK(cudaMemcpyAsync(F.ctrl.p, &hc, sizeof(hc), cudaMemcpyHostToDevice, s));
    F.scale = 1.f;
    if (p->precision == PRT_FP16) {
        const double g0 = std::fabs(p->force) > 0 ? std::fabs(p->force) : 1e-6;
        F.scale = (float)std::ldexp(1.0, (int)std::floor(std::log2(1.0 / g0)));
    }
    fill_lbconst(F.kc, p->nd, p->force, p->tau, p->magic, F.scale);
    F.p = *p;
    F.g = g;
    F.nfluid = nfluid;
    F.d_mat = d_mat;
    F.d_vel = d_vel;
    F.field_ready = false;
    return PRT_OK;
}

int prt::flow_finish(prt_ctx* ctx, prt_flow_info* info) {
    FlowState& F = ctx->flow;
    cudaStream_t s = ctx->stream;
    FlowCtrl res;
    CK(cudaMemcpyAsync(&res, F.ctrl.p, sizeof(res), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // final field from the state after `iters` iterations
    double* parts = F.partials.as<double>();
    CK(flow_launch_moments(F.p.nd, F.p.precision, (res.iters & 1) != 0, F.f.p, F.fm, F.g, F.kc,
                           F.d_vel, parts, s));
    CK(flow_launch_final_reduce(parts, F.nb, F.out5.as<double>(), s));
    ctx->launches += 2;
    double o5[5];
    CK(cudaMemcpyAsync(o5, F.out5.p, sizeof(o5), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (info) {
        memset(info, 0, sizeof(*info));
        info->iters = res.iters;
        info->converged = res.converged;
        info->change = res.change;
        info->fluid_cells = (int64_t)F.nfluid;
        info->ux_sum = o5[0];
        info->mass = o5[1];
        info->speed_sum = o5[2];
        info->umax = o5[3];
        info->nonfinite = (int64_t)llround(o5[4]);
        const double nu = (F.p.tau - 0.5) / 3.0;
        info->permeability =
            F.p.force != 0 ? nu * (o5[0] / (double)F.g.n) / F.p.force : 0.0;
        info->fp16_scale = F.scale;
    }
    F.field_ready = true;
    return PRT_OK;
}

// The flow loop's graph body: `every` step kernels and the convergence
// check (which sets the WHILE condition when h is used).
static cudaError_t flow_emit(prt_ctx* ctx, cudaGraphConditionalHandle h, int use) {
    FlowState& F = ctx->flow;
    const prt_flow_params& p = F.p;
    FlowCtrl* dctrl = F.ctrl.as<FlowCtrl>();
    double* parts = F.partials.as<double>();
    for (int k = 0; k < p.every; ++k) {
        cudaError_t e = flow_launch_step(p.nd, p.precision, (k & 1) != 0, k == p.every - 1,
                                         F.f.p, F.fm, F.g, F.kc, dctrl, k, parts, ctx->stream);
        if (e != cudaSuccess) return e;
    }
    return flow_launch_check(dctrl, parts, F.nb, h, use, ctx->stream);
}

// Builds the loop graph of the set-up flow solve, or reuses the cached one
// when nothing it bakes in has changed.
static int flow_graph(prt_ctx* ctx) {
    FlowState& F = ctx->flow;
    const prt_flow_params& p = F.p;
    FlowKey key;
    key.nd = p.nd; key.precision = p.precision; key.every = p.every; key.g = F.g;
    key.force = p.force; key.tau = p.tau; key.magic = p.magic; key.nit = p.nit;
    key.tol = p.tol; key.f = F.f.p;
    key.aux[0] = F.fluid.p; key.aux[1] = F.partials.p; key.aux[2] = F.ctrl.p;
    key.aux[3] = F.cells.p; key.aux[4] = (void*)F.fm.nbr; key.nf = F.nfluid;
    key.pdl = pdl_key();
    if (!F.graph.exec || !(key == F.key)) {
        CK(build_while_graph(ctx->stream,
                             F.graph, [&](cudaGraphConditionalHandle h, int use) {
                                 return flow_emit(ctx, h, use);
                             }));
        F.key = key;
    }
    return PRT_OK;
}

// Enqueues the whole flow loop of the set-up solve on the context's stream
// without waiting (ev[0] / ev[1] bracket it): one launch of the WHILE graph,
// or every chunk of the plain graph where conditional nodes are missing
// (chunks after the stop are no-ops).
int prt::flow_loop_async(prt_ctx* ctx) {
    FlowState& F = ctx->flow;
    cudaStream_t s = ctx->stream;
    CK(cudaEventRecord(ctx->ev[0], s));
    if (F.p.nit > 0) {
        int rc = flow_graph(ctx);
        if (rc != PRT_OK) return rc;
        const long long chunks = F.graph.conditional ? 1 : (F.p.nit + F.p.every - 1) / F.p.every;
        for (long long r = 0; r < chunks; ++r) CK(cudaGraphLaunch(F.graph.exec, s));
    }
    CK(cudaEventRecord(ctx->ev[1], s));
    return PRT_OK;
}

extern "C" int prt_flow_dev(prt_ctx* ctx, const uint8_t* d_mat, const prt_flow_params* p,
                            float* d_vel, prt_flow_info* info) {
    int rc = flow_setup(ctx, d_mat, p, d_vel);
    if (rc != PRT_OK) return rc;
    FlowState& F = ctx->flow;
    cudaStream_t s = ctx->stream;
    FlowCtrl* dctrl = F.ctrl.as<FlowCtrl>();
    const int every = p->every;
    CK(cudaEventRecord(ctx->ev[0], s));
    if (p->nit > 0) {
        if (graphs_disabled()) {
            // direct launches, chunk by chunk
            FlowCtrl hc2{};
            while (!hc2.done) {
                CK(flow_emit(ctx, cudaGraphConditionalHandle(0), 0));
                ctx->launches += every + 1;
                CK(cudaMemcpyAsync(&hc2, dctrl, sizeof(hc2), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
            }
        } else {
            rc = flow_graph(ctx);
            if (rc != PRT_OK) return rc;
            const long long chunks = (p->nit + every - 1) / every;
            if (F.graph.conditional) {
                CK(cudaGraphLaunch(F.graph.exec, s));
                FlowCtrl hc2;
                CK(cudaMemcpyAsync(&hc2, dctrl, sizeof(hc2), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                ctx->launches += (hc2.iters + every - 1) / every * (every + 1);
            } else {
                FlowCtrl hc2{};
                long long launched = 0;
                while (!hc2.done && launched < chunks) {
                    for (int r = 0; r < 20 && launched < chunks; ++r, ++launched)
                        CK(cudaGraphLaunch(F.graph.exec, s));
                    CK(cudaMemcpyAsync(&hc2, dctrl, sizeof(hc2), cudaMemcpyDeviceToHost, s));
                    CK(cudaStreamSynchronize(s));
                }
                ctx->launches += launched * (every + 1);
            }
        }
    }
    CK(cudaEventRecord(ctx->ev[1], s));
    CK(cudaEventSynchronize(ctx->ev[1]));
    {
        FlowCtrl res;
        CK(cudaMemcpyAsync(&res, dctrl, sizeof(res), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        ctx->timing[0] = ms;
        ctx->timing[1] = (double)res.iters;
    }
    return flow_finish(ctx, info);
}

extern "C" int prt_flow(prt_ctx* ctx, const uint8_t* mat, const prt_flow_params* p, float* vel_out,
                        prt_flow_info* info) {
    if (!ctx || !p || !mat || !vel_out) return fail(ctx, PRT_E_INVALID, "null argument");
    if (p->nd != 2 && p->nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < p->nd; ++i)
        if (p->dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    CK(cudaSetDevice(ctx->device));
    const Grid g = make_grid(p->nd, p->dims);
    FlowState& F = ctx->flow;
    CK(F.mat.ensure((size_t)g.n));
    CK(F.vel.ensure((size_t)g.n * 3 * sizeof(float)));
    CK(cudaMemcpyAsync(F.mat.p, mat, (size_t)g.n, cudaMemcpyHostToDevice, ctx->stream));
    int rc = prt_flow_dev(ctx, F.mat.as<uint8_t>(), p, F.vel.as<float>(), info);
    if (rc != PRT_OK) return rc;
    CK(cudaMemcpyAsync(vel_out, F.vel.p, (size_t)g.n * 3 * sizeof(float), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

// ===========================================================================
// transport
// ===========================================================================
namespace {

struct TreeBuild {
    std::vector<int> leaf_start, leaf_len;
    std::vector<int> in_l, in_r, in_h;  // children encoded: >= 0 leaf id, < 0 -(inner id) - 1
    std::vector<int> leaf_h;
    int build(long long start, long long n) {
        if (n <= 128) {
            leaf_start.push_back((int)start);
            leaf_len.push_back((int)n);
            return (int)leaf_start.size() - 1;
        }
        long long n2 = n / 2;
        n2 -= n2 % 8;
        int l = build(start, n2);
        int r = build(start + n2, n - n2);
        in_l.push_back(l);
        in_r.push_back(r);
        const int hl = l >= 0 ? 0 : in_h[-l - 1];
        const int hr = r >= 0 ? 0 : in_h[-r - 1];
        in_h.push_back(std::max(hl, hr) + 1);
        return -(int)in_l.size();
    }
};

}  // namespace

extern "C" int prt_adr_stage_dev(prt_ctx* ctx, const uint8_t* d_mat, const float* d_vel,
                                 const prt_adr_geom* geom, prt_adr_stats* stats) {
    if (!ctx || !geom || !d_mat || !d_vel) return fail(ctx, PRT_E_INVALID, "null argument");
    if (geom->nd != 2 && geom->nd != 3) return fail(ctx, PRT_E_INVALID, "grid must be 2D or 3D");
    for (int i = 0; i < geom->nd; ++i)
        if (geom->dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    AdrState& A = ctx->adr;
    A.keep_steps.clear();
    A.slot_of_index.clear();
    A.begun = A.ran = false;
    A.staged = false;
    A.geom = *geom;
    const Grid g = make_grid(geom->nd, geom->dims);
    const long long N = g.n;
    A.d.g = g;
    A.d.div_z = make_fastdiv((unsigned)g.nz);
    A.d.div_y = make_fastdiv((unsigned)g.ny);
    A.d.has_bf = geom->biofilm_code >= 0 ? 1 : 0;
    A.d.nd = geom->nd;
    CK(A.flags.ensure((size_t)N * 4));
    CK(A.mflag.ensure((size_t)N));
    A.d.flags = A.flags.as<uint32_t>();
    CK(adr_launch_flags(d_mat, g, geom->nd, geom->pore_code, geom->biofilm_code,
                        A.flags.as<uint32_t>(), A.mflag.as<uint8_t>(), s));
    // compressed solute voxel list
    const int nbs = (int)((N + 1023) / 1024);
    CK(A.cnt.ensure((size_t)nbs * 4));
    CK(A.total.ensure(8));
    CK(adr_launch_compact(A.mflag.as<uint8_t>(), N, A.cnt.as<int>(), A.total.as<long long>(),
                          nullptr, s));
    long long nm = 0;
    CK(cudaMemcpyAsync(&nm, A.total.p, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(A.idx.ensure((size_t)std::max(nm, 1ll) * 4));
    CK(adr_launch_compact(A.mflag.as<uint8_t>(), N, A.cnt.as<int>(), A.total.as<long long>(),
                          A.idx.as<int>(), s));
    ctx->launches += 6;
    A.d.idx = A.idx.as<int>();
    A.d.nm = nm;
    // numpy pairwise tree over nm values
    TreeBuild tb;
    int root = -1;
    if (nm > 0) root = tb.build(0, nm);
    const int L = (int)tb.leaf_start.size();
    const int I = (int)tb.in_l.size();
    // order inner nodes by height
    std::vector<int> order(I);
    for (int i = 0; i < I; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return tb.in_h[a] < tb.in_h[b]; });
    std::vector<int> rank(I);
    for (int r = 0; r < I; ++r) rank[order[r]] = r;
    auto enc = [&](int id) { return id >= 0 ? id : L + rank[-id - 1]; };
    std::vector<int> il(std::max(I, 1)), ir(std::max(I, 1));
    for (int r = 0; r < I; ++r) {
        const int i = order[r];
        il[r] = enc(tb.in_l[i]);
        ir[r] = enc(tb.in_r[i]);
    }
    // inner nodes of height h+1 occupy [loff[h], loff[h+1])
    const int nlevel = I > 0 ? tb.in_h[order[I - 1]] : 0;
    std::vector<int> loff(nlevel + 1, 0);
    for (int r = 0; r < I; ++r) loff[tb.in_h[order[r]]] += 1;
    for (int h = 1; h <= nlevel; ++h) loff[h] += loff[h - 1];
    CK(A.tree_leaf_start.ensure((size_t)std::max(L, 1) * 4));
    CK(A.tree_leaf_len.ensure((size_t)std::max(L, 1) * 4));
    CK(A.tree_inner_l.ensure((size_t)std::max(I, 1) * 4));
    CK(A.tree_inner_r.ensure((size_t)std::max(I, 1) * 4));
    CK(A.tree_level_off.ensure((size_t)(nlevel + 1) * 4));
    CK(A.tree_vals.ensure((size_t)std::max(L + I, 1) * PRT_MAX_SPECIES * 4));
    if (L) {
        CK(cudaMemcpyAsync(A.tree_leaf_start.p, tb.leaf_start.data(), (size_t)L * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(A.tree_leaf_len.p, tb.leaf_len.data(), (size_t)L * 4, cudaMemcpyHostToDevice, s));
    }
    if (I) {
        CK(cudaMemcpyAsync(A.tree_inner_l.p, il.data(), (size_t)I * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(A.tree_inner_r.p, ir.data(), (size_t)I * 4, cudaMemcpyHostToDevice, s));
    }
    CK(cudaMemcpyAsync(A.tree_level_off.p, loff.data(), (size_t)(nlevel + 1) * 4, cudaMemcpyHostToDevice, s));
    // the first leaf of each block of the batch engine (leaves start in order)
    A.nbk = (int)((nm + kBatchAdrBlock - 1) / kBatchAdrBlock);
    std::vector<int> bl((size_t)A.nbk + 1);
    {
        int leaf = 0;
        for (int b = 0; b <= A.nbk; ++b) {
            const long long at = (long long)b * kBatchAdrBlock;
            while (leaf < L && tb.leaf_start[leaf] < at) ++leaf;
            bl[b] = leaf;
        }
    }
    CK(A.blk_leaf.ensure(bl.size() * 4));
    CK(cudaMemcpyAsync(A.blk_leaf.p, bl.data(), bl.size() * 4, cudaMemcpyHostToDevice, s));
    A.d.tree.nleaf = L;
    A.d.tree.ninner = I;
    A.d.tree.nlevel = nlevel;
    A.d.tree.root = nm > 0 ? enc(root) : -1;
    A.d.tree.leaf_start = A.tree_leaf_start.as<int>();
    A.d.tree.leaf_len = A.tree_leaf_len.as<int>();
    A.d.tree.inner_l = A.tree_inner_l.as<int>();
    A.d.tree.inner_r = A.tree_inner_r.as<int>();
    A.d.tree.level_off = A.tree_level_off.as<int>();
    A.d.tree_vals = A.tree_vals.as<float>();
    CK(A.means.ensure(PRT_MAX_SPECIES * 4));
    CK(A.src_slot.ensure(sizeof(float*)));
    CK(A.ctrl.ensure(sizeof(AdrCtrl)));
    // velocity statistics for the host's set-up
    CK(A.tmp.ensure((size_t)N * 4));
    CK(A.vstats.ensure(64));
    CK(cudaMemsetAsync(A.vstats.p, 0, 64, s));
    float* vs_means = A.vstats.as<float>();                                  // 2 floats
    unsigned* vs_max = reinterpret_cast<unsigned*>(A.vstats.as<char>() + 16);  // 3 uints
    unsigned long long* vs_bf = reinterpret_cast<unsigned long long*>(A.vstats.as<char>() + 32);
    CK(adr_launch_vel_stats(d_vel, A.d, A.tmp.as<float>(), vs_means, vs_max, vs_bf, s));
    ctx->launches += 8;
    unsigned char hv[64];
    CK(cudaMemcpyAsync(hv, A.vstats.p, 64, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));  // host vectors above go out of scope
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->solute_voxels = nm;
        memcpy(&stats->biofilm_voxels, hv + 32, 8);
        memcpy(&stats->mean_axial, hv, 4);
        memcpy(&stats->mean_speed, hv + 4, 4);
        memcpy(stats->vmax, hv + 16, 12);
    }
    A.d_mat = d_mat;
    A.d_vel = d_vel;
    A.staged = true;
    return PRT_OK;
}

extern "C" int prt_adr_stage(prt_ctx* ctx, const uint8_t* mat, const float* vel,
                             const prt_adr_geom* geom, prt_adr_stats* stats) {
    if (!ctx || !geom || !mat || !vel) return fail(ctx, PRT_E_INVALID, "null argument");
    if (geom->nd != 2 && geom->nd != 3) return fail(ctx, PRT_E_INVALID, "grid must be 2D or 3D");
    for (int i = 0; i < geom->nd; ++i)
        if (geom->dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    CK(cudaSetDevice(ctx->device));
    const Grid g = make_grid(geom->nd, geom->dims);
    AdrState& A = ctx->adr;
    CK(A.mat.ensure((size_t)g.n));
    CK(A.vel.ensure((size_t)g.n * 3 * 4));
    CK(cudaMemcpyAsync(A.mat.p, mat, (size_t)g.n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(A.vel.p, vel, (size_t)g.n * 3 * 4, cudaMemcpyHostToDevice, ctx->stream));
    return prt_adr_stage_dev(ctx, A.mat.as<uint8_t>(), A.vel.as<float>(), geom, stats);
}

extern "C" int prt_adr_begin(prt_ctx* ctx, const prt_adr_params* p) {
    if (!ctx || !p) return fail(ctx, PRT_E_INVALID, "null argument");
    AdrState& A = ctx->adr;
    if (!A.staged) return fail(ctx, PRT_E_STATE, "prt_adr_begin before prt_adr_stage");
    if (p->nd != A.geom.nd || p->pore_code != A.geom.pore_code ||
        p->biofilm_code != A.geom.biofilm_code)
        return fail(ctx, PRT_E_INVALID, "parameters do not match the staged geometry");
    for (int i = 0; i < p->nd; ++i)
        if (p->dims[i] != A.geom.dims[i])
            return fail(ctx, PRT_E_INVALID, "parameters do not match the staged geometry");
    if (p->ns < 1 || p->ns > PRT_MAX_SPECIES)
        return fail(ctx, PRT_E_INVALID, "between 1 and 8 chemicals are supported");
    if (!(p->dt > 0.f)) return fail(ctx, PRT_E_INVALID, "the time step must be positive");
    if ((long long)p->ns * (A.d.g.n + A.d.g.n / std::max(1, A.d.g.nx) + 1) >= (1ll << 31))
        return fail(ctx, PRT_E_INVALID,
                    "chemicals x voxels too large for the transport's 32-bit indices");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    A.p = *p;
    const Grid g = A.d.g;
    const long long N = g.n;
    A.d.ns = p->ns;
    for (int a = 0; a < 3; ++a) {
        const int ext = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
        const bool active = (p->nd == 3) || a != 1;
        CK(A.face[a].ensure(active ? (size_t)(N / ext * (ext + 1)) * 4 : 4));
        A.d.face[a] = A.face[a].as<float>();
    }
    CK(A.buf[0].ensure((size_t)N * p->ns * 4));
    CK(A.buf[1].ensure((size_t)N * p->ns * 4));
    CK(cudaMemsetAsync(A.buf[1].p, 0, (size_t)N * p->ns * 4, s));
    A.d.buf[0] = A.buf[0].as<float>();
    A.d.buf[1] = A.buf[1].as<float>();
    A.d.ladder = nullptr;  // allocated by prt_adr_run
    CK(adr_launch_setup(A.d_mat, A.d_vel, *p, A.d, s));
    ctx->launches += p->nd + 1;
    CK(cudaStreamSynchronize(s));
    A.begun = true;
    A.ran = false;
    return PRT_OK;
}

// Transport time loop in three parts (see flow_setup): the ladder and the
// control block, the loop, and the kept snapshots.
int prt::adr_run_setup(prt_ctx* ctx, const prt_adr_run_params* rp, long long pause_every) {
    if (!ctx || !rp) return fail(ctx, PRT_E_INVALID, "null argument");
    AdrState& A = ctx->adr;
    if (!A.begun) return fail(ctx, PRT_E_STATE, "prt_adr_run before prt_adr_begin");
    if (rp->limit < 0 || rp->check <= 0 || !(rp->ratio > 0))
        return fail(ctx, PRT_E_INVALID, "bad run parameters");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const long long N = A.d.g.n;
    const int ns = A.p.ns;
    const long long limit = rp->limit;
    // the snapshot ladder (prtlb_3d.py:1496-1498): record at n >= nxt,
    // nxt = max(n + 1, ceil(n * ratio)); steps are known before the run
    A.sched.clear();
    {
        long long nxt = 1;
        for (long long n = nxt; n <= limit;) {
            A.sched.push_back(n);
            long long c2 = (long long)std::ceil((double)n * rp->ratio);
            nxt = std::max(n + 1, c2);
            n = nxt;
        }
    }
    const int K = (int)A.sched.size();
    A.nslots = K + 2;  // step 0, the schedule, and a final record
    const size_t slot_bytes = (size_t)N * ns * 4;
    CK(A.ladder.ensure(slot_bytes * A.nslots));
    CK(cudaMemsetAsync(A.ladder.p, 0, slot_bytes * A.nslots, s));
    CK(cudaMemcpyAsync(A.ladder.p, A.buf[0].p, slot_bytes, cudaMemcpyDeviceToDevice, s));
    std::vector<int> sos((size_t)limit + 1, -1);
    for (int k = 0; k < K; ++k) sos[(size_t)A.sched[k]] = k + 1;
    CK(A.slot_of_step.ensure(sos.size() * 4));
    CK(cudaMemcpyAsync(A.slot_of_step.p, sos.data(), sos.size() * 4, cudaMemcpyHostToDevice, s));
    const int log_cap = (int)(limit / rp->check) + 2;
    CK(A.log.ensure((size_t)log_cap * sizeof(ProgressRec)));
    A.d.ladder = A.ladder.as<float>();
    A.d.slot_of_step = A.slot_of_step.as<int>();
    A.d.log = A.log.as<ProgressRec>();
    A.d.log_cap = log_cap;

    AdrCtrl hc{};
    hc.n_base = 0;
    hc.limit = limit;
    hc.check = rp->check;
    hc.until_conv = rp->until_conv;
    hc.tol = rp->tol;
    hc.ns = ns;
    hc.last_rest = INFINITY;
    for (int j = 0; j < PRT_MAX_SPECIES; ++j) {
        hc.prev[j] = 0.0;
        hc.prev_change[j] = 0.0;
        hc.scale[j] = 1e-6;
    }
    hc.n_pause = std::min(limit, pause_every);
    hc.done = limit == 0 ? 1 : 0;
    CK(cudaMemcpyAsync(A.ctrl.p, &hc, sizeof(hc), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));  // the host vector above goes out of scope
    A.rp = *rp;
    return PRT_OK;
}

int prt::adr_run_finish(prt_ctx* ctx, prt_adr_result* res) {
    AdrState& A = ctx->adr;
    cudaStream_t s = ctx->stream;
    AdrCtrl cur;
    CK(cudaMemcpyAsync(&cur, A.ctrl.p, sizeof(cur), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const long long n = cur.n_base;
    const int K = (int)A.sched.size();
    const size_t slot_bytes = (size_t)A.d.g.n * A.p.ns * 4;
    // keep_steps = [0] + ladder steps <= n, plus n itself when not one of them
    A.keep_steps.clear();
    A.slot_of_index.clear();
    A.keep_steps.push_back(0);
    A.slot_of_index.push_back(0);
    for (int k = 0; k < K && A.sched[k] <= n; ++k) {
        A.keep_steps.push_back(A.sched[k]);
        A.slot_of_index.push_back(k + 1);
    }
    if (A.keep_steps.back() != n) {
        CK(cudaMemcpyAsync(A.ladder.as<char>() + slot_bytes * (K + 1), A.buf[n & 1].p, slot_bytes,
                           cudaMemcpyDeviceToDevice, s));
        A.keep_steps.push_back(n);
        A.slot_of_index.push_back(K + 1);
    }
    CK(cudaStreamSynchronize(s));
    A.ran = true;
    if (res) {
        memset(res, 0, sizeof(*res));
        res->steps = n;
        res->hit_cap = (A.rp.until_conv && n >= A.rp.limit) ? 1 : 0;
        res->ladder = (int32_t)A.keep_steps.size();
        res->checks = cur.checks;
        res->last_rest = cur.last_rest;
    }
    return PRT_OK;
}

// The transport loop's graph body: `check` step kernels, the numpy-order
// means of the chunk's last step and the stop rule (which sets the WHILE
// condition when h is used).
static cudaError_t adr_emit(prt_ctx* ctx, cudaGraphConditionalHandle h, int use) {
    AdrState& A = ctx->adr;
    AdrCtrl* dctrl = A.ctrl.as<AdrCtrl>();
    float* dmeans = A.means.as<float>();
    const float** srcp = (const float**)A.src_slot.p;
    for (int k = 0; k < A.rp.check; ++k) {
        cudaError_t e = adr_launch_step(A.d, A.p, dctrl, k, ctx->stream);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = adr_launch_chunk_means(A.d, dctrl, srcp, dmeans, ctx->stream);
    if (e != cudaSuccess) return e;
    return adr_launch_stop(A.d, dctrl, dmeans, h, use, ctx->stream);
}

// Everything the transport loop graph bakes into its nodes: the device
// descriptor and parameters the step kernels take by value, the chunk length,
// the buffers of the means and the stop rule, and the launch attribute.
static std::vector<unsigned char> adr_graph_key(prt_ctx* ctx) {
    AdrState& A = ctx->adr;
    const void* ptrs[3] = {A.means.p, A.src_slot.p, A.ctrl.p};
    const int ints[2] = {A.rp.check, pdl_key()};
    std::vector<unsigned char> k(sizeof(AdrDev) + sizeof(prt_adr_params) + sizeof(ptrs) +
                                 sizeof(ints));
    unsigned char* q = k.data();
    memcpy(q, &A.d, sizeof(AdrDev));
    q += sizeof(AdrDev);
    memcpy(q, &A.p, sizeof(prt_adr_params));
    q += sizeof(prt_adr_params);
    memcpy(q, ptrs, sizeof(ptrs));
    q += sizeof(ptrs);
    memcpy(q, ints, sizeof(ints));
    return k;
}

// The loop graph of the set-up run: the cached one when the key matches
// (back-to-back solves of one geometry and chemistry), else a new capture.
static cudaError_t adr_graph(prt_ctx* ctx) {
    AdrState& A = ctx->adr;
    std::vector<unsigned char> key = adr_graph_key(ctx);
    if (A.graph.exec && key == A.graph_key) return cudaSuccess;
    A.graph_key.clear();
    cudaError_t e = build_while_graph(ctx->stream, A.graph, [&](cudaGraphConditionalHandle h,
                                                                int use) {
        return adr_emit(ctx, h, use);
    });
    if (e == cudaSuccess) A.graph_key = key;
    return e;
}

// Enqueues the whole transport loop of a started run (adr_run_setup with no
// pause) without waiting (ev[2] / ev[3] bracket it), as flow_loop_async.
int prt::adr_loop_async(prt_ctx* ctx) {
    AdrState& A = ctx->adr;
    cudaStream_t s = ctx->stream;
    CK(cudaEventRecord(ctx->ev[2], s));
    if (A.rp.limit > 0) {
        CK(adr_graph(ctx));
        const long long chunks =
            A.graph.conditional ? 1 : (A.rp.limit + A.rp.check - 1) / A.rp.check;
        for (long long r = 0; r < chunks; ++r) CK(cudaGraphLaunch(A.graph.exec, s));
    }
    CK(cudaEventRecord(ctx->ev[3], s));
    return PRT_OK;
}

extern "C" int prt_adr_run(prt_ctx* ctx, const prt_adr_run_params* rp, prt_progress_cb cb,
                           void* user, prt_adr_result* res) {
    if (!ctx || !rp) return fail(ctx, PRT_E_INVALID, "null argument");
    // with a progress callback the host regains control every few checks
    const long long pause_every = cb ? (long long)rp->check * 8 : rp->limit;
    int rc = adr_run_setup(ctx, rp, pause_every);
    if (rc != PRT_OK) return rc;
    AdrState& A = ctx->adr;
    cudaStream_t s = ctx->stream;
    const long long limit = rp->limit;
    const int log_cap = A.d.log_cap;
    AdrCtrl* dctrl = A.ctrl.as<AdrCtrl>();
    const int check = rp->check;
    const AdrDev D = A.d;
    auto emit = [&](cudaGraphConditionalHandle h, int use) -> cudaError_t {
        return adr_emit(ctx, h, use);
    };
    const int per_chunk = check + 3 + (D.tree.nleaf > 0 ? 1 : 0);
    std::vector<ProgressRec> logbuf;
    int delivered = 0;
    AdrCtrl cur;
    CK(cudaMemcpyAsync(&cur, dctrl, sizeof(cur), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    bool use_graph = !graphs_disabled();
    if (use_graph && !cur.done) CK(adr_graph(ctx));
    CK(cudaEventRecord(ctx->ev[2], s));
    while (!cur.done) {
        if (!use_graph) {
            CK(emit(cudaGraphConditionalHandle(0), 0));
            ctx->launches += per_chunk;
        } else if (A.graph.conditional) {
            CK(cudaGraphLaunch(A.graph.exec, s));
        } else {
            for (int r = 0; r < 4; ++r) {
                CK(cudaGraphLaunch(A.graph.exec, s));
                ctx->launches += per_chunk;
            }
        }
        const long long before = cur.n_base;
        CK(cudaMemcpyAsync(&cur, dctrl, sizeof(cur), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (use_graph && A.graph.conditional)
            ctx->launches += (cur.n_base - before + check - 1) / check * per_chunk;
        if (cb && cur.nlog > delivered) {
            const int nrec = std::min(cur.nlog, log_cap) - delivered;
            logbuf.resize(nrec);
            if (nrec > 0) {
                CK(cudaMemcpy(logbuf.data(), A.d.log + delivered, nrec * sizeof(ProgressRec),
                              cudaMemcpyDeviceToHost));
            }
            for (int i = 0; i < nrec; ++i) {
                if (cb(user, logbuf[i].n, limit, logbuf[i].mean0, logbuf[i].value) != 0) {
                    A.ran = true;
                    return fail(ctx, PRT_E_CANCELLED, "cancelled by the progress callback");
                }
            }
            delivered += nrec;
        }
        if (!cur.done && cur.n_base >= cur.n_pause) {
            cur.n_pause = std::min(limit, cur.n_pause + pause_every);
            CK(cudaMemcpyAsync(&dctrl->n_pause, &cur.n_pause, sizeof(long long),
                               cudaMemcpyHostToDevice, s));
        }
    }
    CK(cudaEventRecord(ctx->ev[3], s));
    CK(cudaEventSynchronize(ctx->ev[3]));
    {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
        ctx->timing[2] = ms;
        ctx->timing[3] = (double)cur.n_base;
    }
    return adr_run_finish(ctx, res);
}

extern "C" int prt_adr_ladder(prt_ctx* ctx, int64_t* steps, int32_t cap, int32_t* count) {
    if (!ctx) return PRT_E_INVALID;
    AdrState& A = ctx->adr;
    if (!A.ran) return fail(ctx, PRT_E_STATE, "no finished run");
    const int n = (int)A.keep_steps.size();
    if (count) *count = n;
    if (steps)
        for (int i = 0; i < n && i < cap; ++i) steps[i] = A.keep_steps[i];
    return PRT_OK;
}

static int slot_ptr(prt_ctx* ctx, int32_t slot, const float** out) {
    AdrState& A = ctx->adr;
    if (!A.ran) return fail(ctx, PRT_E_STATE, "no finished run");
    if (slot < 0 || slot >= (int)A.slot_of_index.size())
        return fail(ctx, PRT_E_INVALID, "snapshot index out of range");
    *out = A.ladder.as<float>() + (size_t)A.slot_of_index[slot] * A.d.g.n * A.p.ns;
    return PRT_OK;
}

extern "C" int prt_adr_fetch(prt_ctx* ctx, int32_t slot, float* out) {
    if (!ctx || !out) return fail(ctx, PRT_E_INVALID, "null argument");
    const float* src = nullptr;
    int rc = slot_ptr(ctx, slot, &src);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)ctx->adr.d.g.n * ctx->adr.p.ns * 4;
    CK(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

extern "C" int prt_adr_fetch_dev(prt_ctx* ctx, int32_t slot, float* d_out) {
    if (!ctx || !d_out) return fail(ctx, PRT_E_INVALID, "null argument");
    const float* src = nullptr;
    int rc = slot_ptr(ctx, slot, &src);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)ctx->adr.d.g.n * ctx->adr.p.ns * 4;
    CK(cudaMemcpyAsync(d_out, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

extern "C" int prt_adr_means(prt_ctx* ctx, int32_t slot, float* means) {
    if (!ctx || !means) return fail(ctx, PRT_E_INVALID, "null argument");
    AdrState& A = ctx->adr;
    if (!A.ran) return fail(ctx, PRT_E_STATE, "no finished run");
    if (slot < 0 || slot >= (int)A.slot_of_index.size())
        return fail(ctx, PRT_E_INVALID, "snapshot index out of range");
    CK(cudaSetDevice(ctx->device));
    CK(adr_launch_means(A.d, A.ctrl.as<AdrCtrl>(), A.slot_of_index[slot], A.means.as<float>(),
                        ctx->stream));
    ctx->launches += 2;
    CK(cudaMemcpyAsync(means, A.means.p, (size_t)A.p.ns * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

// Transport buffers up to this size outlive prt_adr_end on their context.
constexpr size_t kAdrKeepBytes = size_t(256) << 20;

extern "C" int prt_adr_end(prt_ctx* ctx) {
    if (!ctx) return PRT_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->adr.release(kAdrKeepBytes);
    return PRT_OK;
}

extern "C" int prt_adr_release(prt_ctx* ctx) {
    if (!ctx) return PRT_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->adr.release();
    return PRT_OK;
}
