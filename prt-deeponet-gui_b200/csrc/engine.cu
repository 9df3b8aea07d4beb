// engine.cu -- batched and served solves: the split single-solve entry points
// (start / finish) and the batch engine that runs the time loops of many
// started solves together.
//
// A batch keeps a list of contexts, each in its flow loop or in its transport
// loop.  Every batch step advances each of them by one iteration (flow) or
// one step (transport): one persistent launch per class of jobs -- (lattice,
// precision) for flow, (dimension, species) for transport -- walks a work
// list of voxel tiles of all jobs of the class.  Each class's chain of
// launches is captured on its own stream, so the classes overlap in the
// graph.  Work
// lists, job descriptors and counts live in device memory and the launches
// read their lengths there, so a graph stays valid while jobs come and go;
// it is rebuilt only when the set of classes, a grid size or a buffer
// address changes.
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "runtime_internal.h"

using namespace prt;

namespace {

constexpr int kFlowClasses = 8;  // (nd 2|3) x 4 precisions
constexpr int kAdrClasses = 16;  // (nd 2|3) x species 1..8
constexpr int kClasses = kFlowClasses + kAdrClasses;
constexpr int kCounts = kClasses;  // counts[]: tiles per class

int flow_class(int nd, int precision) { return (nd == 3 ? 4 : 0) + precision; }
int adr_class(int nd, int ns) { return kFlowClasses + (nd == 3 ? 8 : 0) + (ns - 1); }

// Growable device buffer whose address changes only when it grows.
struct GrowBuf {
    DevBuf b;
    cudaError_t fit(size_t bytes) {
        if (bytes <= b.bytes && b.p) return cudaSuccess;
        size_t want = std::max<size_t>(bytes, 256);
        want = std::max(want, b.bytes * 2);
        return b.ensure(want);
    }
};

struct Candidate {
    int tile_blocks;
    int grid_mult;
};
// grid_mult 0: one block per work-list entry (no persistent loop)
const Candidate kCandidates[] = {{1, 0}, {1, 1}, {2, 1}, {4, 0}};
constexpr int kNumCandidates = 4;
// launches timed per candidate; its cost is the cheapest of them (the first
// launch after a rebuild also uploads the new graph)
constexpr int kTunePasses = 2;
// the candidates are timed again when the flow solves' share of the work
// has moved this far from the share they were timed on (the best tiling of
// a batch of flow solves is not that of a batch of transport runs), or the
// work itself has grown or shrunk by this factor (few blocks want one block
// per tile, many want longer tiles)
constexpr double kRetuneShift = 0.3;
constexpr double kRetuneScale = 1.5;

}  // namespace

struct prt_batch {
    int device = 0;
    int nsm = 148;
    int K = 20;  // steps per graph replay
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    // one stream per class while a graph is captured: the classes' chains
    // are independent (no job is in two classes), so they run side by side
    cudaStream_t cls_stream[kClasses] = {};
    cudaEvent_t cls_join[kClasses] = {};
    std::string err;
    std::mutex mu;
    std::vector<prt_ctx*> jobs;  // in the batch
    bool dirty = true;
    // what the last rebuild uploaded
    std::vector<prt_ctx*> order;  // flow jobs then transport jobs (status order)
    int nflow = 0, nadr = 0;
    std::vector<FlowJob> h_flow;
    std::vector<AdrJob> h_adr;
    std::vector<const int*> h_done;
    std::vector<BatchTile> h_tiles[kClasses];
    int h_counts[kCounts] = {};
    int grid[kClasses] = {};
    // flow classes whose jobs all share their constants (passed as a parameter)
    bool flow_uni[kFlowClasses] = {};
    LbParams flow_kc[kFlowClasses] = {};
    GrowBuf d_flow, d_adr, d_done, d_status, d_arrive, d_adr_cnt, d_counts;
    GrowBuf d_gstep;  // batch steps done (one long long), advanced by each replay
    GrowBuf d_tiles[kClasses];
    int* h_status = nullptr;  // pinned
    size_t h_status_cap = 0;
    // graph
    GraphHolder graph;
    std::vector<long long> graph_key;
    // tiling
    int tile_blocks = 1, grid_mult = 1;
    bool auto_tile = true, tuning = true;
    int cand = 0, cand_pass = 0;
    double cand_cost[kNumCandidates] = {};
    double tune_share = -1.0;  // flow share of the work the tiling was timed on
    long long tune_blocks = 0;  // and its blocks
    // the launch in flight
    bool in_flight = false;
    int launch_replays = 0;
    long long launch_blocks = 0;
    // statistics
    int64_t launches = 0, graph_builds = 0, steps_run = 0;
    double last_ms = 0;
    long long last_tiles = 0;
};

namespace {

int bfail(prt_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    return code;
}

int bcuda(prt_batch* b, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return bfail(b, e == cudaErrorMemoryAllocation ? PRT_E_OOM : PRT_E_CUDA, m);
}

#define BK(expr)                                                 \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return bcuda(b, _e, #expr);       \
    } while (0)

bool is_flow_job(const prt_ctx* c) { return c->flow_armed; }

// The flow solves' share of the batch's blocks of work, and their number.
double flow_share(const prt_batch* b, long long* blocks = nullptr) {
    long long fl = 0, all = 0;
    for (const prt_ctx* c : b->jobs) {
        const long long n = is_flow_job(c) ? c->flow.nb : c->adr.nbk;
        all += n;
        if (is_flow_job(c)) fl += n;
    }
    if (blocks) *blocks = all;
    return all ? (double)fl / (double)all : 0.0;
}

// The g0 of a job (see FlowJob): fixed at the first launch after it joined,
// from the batch steps done then and the count it joined with.
long long job_g0(prt_batch* b, prt_ctx* c) {
    if (!c->batch_g0_set) {
        c->batch_g0 = b->steps_run - c->batch_c0;
        c->batch_g0_set = true;
    }
    return c->batch_g0;
}

// Job lists, work lists and grids for the current jobs; uploads them.
int rebuild(prt_batch* b) {
    b->order.clear();
    b->h_flow.clear();
    b->h_adr.clear();
    b->h_done.clear();
    for (int c = 0; c < kClasses; ++c) b->h_tiles[c].clear();
    for (prt_ctx* c : b->jobs)
        if (is_flow_job(c)) b->order.push_back(c);
    b->nflow = (int)b->order.size();
    for (prt_ctx* c : b->jobs)
        if (!is_flow_job(c)) b->order.push_back(c);
    b->nadr = (int)b->order.size() - b->nflow;
    const int T = b->tile_blocks;
    long long blocks = 0;
    size_t adr_cnt = 0;  // transport counters: per job, arrival + seams
    for (int i = 0; i < b->nflow; ++i) {
        prt_ctx* c = b->order[i];
        FlowState& F = c->flow;
        FlowJob J{};
        J.f = F.f.p;
        J.fm = F.fm;
        J.g = F.g;
        J.kc = F.kc;
        J.ctrl = F.ctrl.as<FlowCtrl>();
        J.partials = F.partials.as<double>();
        J.arrive = nullptr;  // set after the counter array is sized
        J.nb = F.nb;
        J.g0 = job_g0(b, c);
        b->h_flow.push_back(J);
        const int cls = flow_class(F.p.nd, F.p.precision);
        for (int b0 = 0; b0 < F.nb; b0 += T)
            b->h_tiles[cls].push_back(BatchTile{i, b0, std::min(T, F.nb - b0), 0});
        blocks += F.nb;
        b->h_done.push_back(&J.ctrl->done);
    }
    for (int i = 0; i < b->nadr; ++i) {
        prt_ctx* c = b->order[b->nflow + i];
        AdrState& A = c->adr;
        AdrJob J{};
        J.d = A.d;
        J.p = A.p;
        J.ctrl = A.ctrl.as<AdrCtrl>();
        J.means = A.means.as<float>();
        J.cnt = nullptr;  // set after the counter array is sized
        J.blk_leaf = A.blk_leaf.as<const int>();
        J.nbk = A.nbk;
        J.g0 = job_g0(b, c);
        b->h_adr.push_back(J);
        const int cls = adr_class(A.d.nd, A.d.ns);
        const int nbk = A.nbk;
        for (int b0 = 0; b0 < nbk; b0 += T)
            b->h_tiles[cls].push_back(BatchTile{i, b0, std::min(T, nbk - b0), 0});
        // a run without solute voxels still steps (its control block
        // advances) through one empty tile
        if (nbk == 0) b->h_tiles[cls].push_back(BatchTile{i, 0, 0, 0});
        blocks += nbk;
        adr_cnt += (size_t)nbk + 1;
        b->h_done.push_back(&J.ctrl->done);
    }
    // pull tables: each solve chose them against the whole L2 cache; in a
    // batch they pay only while the flow jobs' lattices and tables together
    // fit in half of it, otherwise the tables' bytes add to the DRAM traffic
    // and the kernels look the upstream slots up through the maps (the same
    // slots either way, so the fields do not change)
    {
        long long ws = 0, l2 = 0;
        for (int i = 0; i < b->nflow; ++i) {
            const prt_ctx* c = b->order[i];
            const FlowState& F = c->flow;
            const int q = F.p.nd == 3 ? 19 : 9;
            const long long es = F.p.precision == PRT_FP64 ? 8 : F.p.precision == PRT_FP16 ? 2 : 4;
            ws += 2ll * q * F.fm.nf * es + (F.fm.nbr ? flow_nbr_bytes(q, F.fm.nf) / 2 : 0);
            l2 = c->l2_bytes;
        }
        const char* v = std::getenv("PRT_NBR_TABLE");
        const bool forced = v && v[0] == '1';
        if (!forced && ws > l2 / 2)
            for (FlowJob& J : b->h_flow) J.fm.nbr = nullptr;
    }
    for (int c = 0; c < kFlowClasses; ++c) b->flow_uni[c] = false;
    {
        bool seen[kFlowClasses] = {}, differ[kFlowClasses] = {};
        for (int i = 0; i < b->nflow; ++i) {
            const FlowState& F = b->order[i]->flow;
            const int c = flow_class(F.p.nd, F.p.precision);
            if (!seen[c]) {
                seen[c] = true;
                b->flow_kc[c] = b->h_flow[i].kc;
            } else if (std::memcmp(&b->flow_kc[c], &b->h_flow[i].kc, sizeof(LbParams)) != 0) {
                differ[c] = true;
            }
        }
        for (int c = 0; c < kFlowClasses; ++c) b->flow_uni[c] = seen[c] && !differ[c];
    }
    const int njobs = (int)b->order.size();
    BK(b->d_arrive.fit((size_t)std::max(b->nflow, 1) * sizeof(unsigned)));
    for (int i = 0; i < b->nflow; ++i) b->h_flow[i].arrive = b->d_arrive.b.as<unsigned>() + i;
    BK(b->d_adr_cnt.fit(std::max<size_t>(adr_cnt, 1) * sizeof(unsigned)));
    {
        unsigned* at = b->d_adr_cnt.b.as<unsigned>();
        for (AdrJob& J : b->h_adr) {
            J.cnt = at;
            at += J.nbk + 1;
        }
    }
    BK(b->d_flow.fit(std::max<size_t>(b->h_flow.size(), 1) * sizeof(FlowJob)));
    BK(b->d_adr.fit(std::max<size_t>(b->h_adr.size(), 1) * sizeof(AdrJob)));
    BK(b->d_done.fit((size_t)std::max(njobs, 1) * sizeof(int*)));
    BK(b->d_status.fit((size_t)std::max(njobs, 1) * sizeof(int)));
    BK(b->d_counts.fit(kCounts * sizeof(int)));
    if ((size_t)njobs > b->h_status_cap) {
        if (b->h_status) cudaFreeHost(b->h_status);
        b->h_status = nullptr;
        b->h_status_cap = 0;
        BK(cudaMallocHost(&b->h_status, (size_t)std::max(njobs, 64) * 2 * sizeof(int)));
        b->h_status_cap = (size_t)std::max(njobs, 64) * 2;
    }
    cudaStream_t s = b->stream;
    for (int c = 0; c < kClasses; ++c) {
        b->h_counts[c] = (int)b->h_tiles[c].size();
        BK(b->d_tiles[c].fit(std::max<size_t>(b->h_tiles[c].size(), 1) * sizeof(BatchTile)));
        if (!b->h_tiles[c].empty())
            BK(cudaMemcpyAsync(b->d_tiles[c].b.p, b->h_tiles[c].data(),
                               b->h_tiles[c].size() * sizeof(BatchTile), cudaMemcpyHostToDevice, s));
    }
    if (!b->h_flow.empty())
        BK(cudaMemcpyAsync(b->d_flow.b.p, b->h_flow.data(), b->h_flow.size() * sizeof(FlowJob),
                           cudaMemcpyHostToDevice, s));
    if (!b->h_adr.empty())
        BK(cudaMemcpyAsync(b->d_adr.b.p, b->h_adr.data(), b->h_adr.size() * sizeof(AdrJob),
                           cudaMemcpyHostToDevice, s));
    if (njobs)
        BK(cudaMemcpyAsync(b->d_done.b.p, b->h_done.data(), (size_t)njobs * sizeof(int*),
                           cudaMemcpyHostToDevice, s));
    BK(cudaMemcpyAsync(b->d_counts.b.p, b->h_counts, sizeof(b->h_counts), cudaMemcpyHostToDevice, s));
    BK(cudaMemsetAsync(b->d_arrive.b.p, 0, (size_t)std::max(b->nflow, 1) * sizeof(unsigned), s));
    BK(cudaMemsetAsync(b->d_adr_cnt.b.p, 0, std::max<size_t>(adr_cnt, 1) * sizeof(unsigned), s));
    // the host vectors must outlive the copies
    BK(cudaStreamSynchronize(s));
    // persistent grids: grid_mult resident waves, at most one block per tile
    for (int c = 0; c < kClasses; ++c) {
        const int nt = b->h_counts[c];
        if (!nt) {
            b->grid[c] = 0;
            continue;
        }
        int occ = 1;
        if (c < kFlowClasses) occ = batch_flow_occupancy(c >= 4 ? 3 : 2, c % 4);
        else occ = batch_adr_occupancy(c >= kFlowClasses + 8 ? 3 : 2, (c - kFlowClasses) % 8 + 1);
        b->grid[c] = b->grid_mult == 0 ? nt
                                       : std::max(1, std::min(nt, b->grid_mult * occ * b->nsm));
    }
    b->launch_blocks = blocks;
    b->last_tiles = 0;
    for (int c = 0; c < kClasses; ++c) b->last_tiles += b->h_counts[c];
    b->dirty = false;
    return PRT_OK;
}

// One batch step: the launch of class c on streams[c], or on `s` for every
// class when streams is null.
cudaError_t emit_step(prt_batch* b, cudaStream_t s, const cudaStream_t* streams, int k) {
    const int* counts = b->d_counts.b.as<int>();
    for (int c = 0; c < kClasses; ++c) {
        if (!b->grid[c]) continue;
        cudaStream_t sc = streams ? streams[c] : s;
        cudaError_t e;
        if (c < kFlowClasses) {
            e = batch_launch_flow(c >= 4 ? 3 : 2, c % 4, b->d_flow.b.as<FlowJob>(),
                                  b->d_tiles[c].b.as<BatchTile>(), counts + c,
                                  b->d_gstep.b.as<long long>(), k,
                                  b->flow_uni[c] ? &b->flow_kc[c] : nullptr, b->grid[c], sc);
        } else {
            const int a = c - kFlowClasses;
            e = batch_launch_adr(a >= 8 ? 3 : 2, a % 8 + 1, b->d_adr.b.as<AdrJob>(),
                                 b->d_tiles[c].b.as<BatchTile>(), counts + c,
                                 b->d_gstep.b.as<long long>(), k, b->grid[c], sc);
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int launches_per_step(const prt_batch* b) {
    int n = 0;
    for (int c = 0; c < kClasses; ++c) n += b->grid[c] ? 1 : 0;
    return n;
}

// Graph of K steps: each class's chain of K launches on its own stream,
// forked from and joined back to the batch stream.
int ensure_graph(prt_batch* b) {
    std::vector<long long> key;
    key.push_back(b->K);
    for (int c = 0; c < kClasses; ++c) key.push_back(b->grid[c]);
    for (int c = 0; c < kFlowClasses; ++c) {  // constants baked into the launches
        key.push_back(b->flow_uni[c]);
        if (!b->flow_uni[c]) continue;
        long long w[(sizeof(LbParams) + 7) / 8] = {};
        std::memcpy(w, &b->flow_kc[c], sizeof(LbParams));
        for (long long x : w) key.push_back(x);
    }
    key.push_back((long long)b->d_flow.b.p);
    key.push_back((long long)b->d_adr.b.p);
    key.push_back((long long)b->d_counts.b.p);
    for (int c = 0; c < kClasses; ++c) key.push_back((long long)b->d_tiles[c].b.p);
    if (b->graph.exec && key == b->graph_key) return PRT_OK;
    b->graph.release();
    for (int c = 0; c < kClasses; ++c) {
        if (!b->grid[c] || b->cls_stream[c]) continue;
        BK(cudaStreamCreateWithFlags(&b->cls_stream[c], cudaStreamNonBlocking));
        BK(cudaEventCreateWithFlags(&b->cls_join[c], cudaEventDisableTiming));
    }
    cudaStream_t s = b->stream;
    BK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaEventRecord(b->fork, s);
    for (int c = 0; c < kClasses && e == cudaSuccess; ++c)
        if (b->grid[c]) e = cudaStreamWaitEvent(b->cls_stream[c], b->fork, 0);
    for (int k = 0; k < b->K && e == cudaSuccess; ++k) e = emit_step(b, s, b->cls_stream, k);
    for (int c = 0; c < kClasses && e == cudaSuccess; ++c) {
        if (!b->grid[c]) continue;
        e = cudaEventRecord(b->cls_join[c], b->cls_stream[c]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->cls_join[c], 0);
    }
    if (e == cudaSuccess) e = batch_launch_gstep(b->d_gstep.b.as<long long>(), b->K, s);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return bcuda(b, e, "batch graph capture");
    }
    if (e2 != cudaSuccess) return bcuda(b, e2, "cudaStreamEndCapture");
    b->graph.graph = g;
    BK(cudaGraphInstantiate(&b->graph.exec, g, 0));
    b->graph_key = key;
    b->graph_builds += 1;
    return PRT_OK;
}

}  // namespace

void prt::batch_detach(prt_ctx* c) {
    prt_batch* b = c ? c->batch : nullptr;
    if (!b) return;
    std::lock_guard<std::mutex> lk(b->mu);
    auto it = std::find(b->jobs.begin(), b->jobs.end(), c);
    if (it != b->jobs.end()) b->jobs.erase(it);
    for (auto& o : b->order)
        if (o == c) o = nullptr;
    b->dirty = true;
    c->batch = nullptr;
    c->batch_g0_set = false;
}

// ===========================================================================
// split single solves
// ===========================================================================
extern "C" int prt_flow_start(prt_ctx* ctx, const uint8_t* mat, const prt_flow_params* p) {
    if (!ctx || !p || !mat) return fail(ctx, PRT_E_INVALID, "null argument");
    if (ctx->batch) return fail(ctx, PRT_E_STATE, "the context is in a batch");
    if (p->nd != 2 && p->nd != 3) return fail(ctx, PRT_E_INVALID, "nd must be 2 or 3");
    for (int i = 0; i < p->nd; ++i)
        if (p->dims[i] <= 0) return fail(ctx, PRT_E_INVALID, "grid dimensions must be positive");
    CK(cudaSetDevice(ctx->device));
    const Grid g = make_grid(p->nd, p->dims);
    FlowState& F = ctx->flow;
    CK(F.mat.ensure((size_t)g.n));
    CK(F.vel.ensure((size_t)g.n * 3 * sizeof(float)));
    CK(cudaMemcpyAsync(F.mat.p, mat, (size_t)g.n, cudaMemcpyHostToDevice, ctx->stream));
    ctx->flow_armed = false;
    int rc = flow_setup(ctx, F.mat.as<uint8_t>(), p, F.vel.as<float>());
    if (rc != PRT_OK) return rc;
    // the batch runs on another stream: the set-up must be complete
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->flow_armed = true;
    return PRT_OK;
}

extern "C" int prt_flow_finish(prt_ctx* ctx, float* vel_out, prt_flow_info* info) {
    if (!ctx) return PRT_E_INVALID;
    if (ctx->batch) return fail(ctx, PRT_E_STATE, "the context is in a batch");
    if (!ctx->flow_armed) return fail(ctx, PRT_E_STATE, "no started flow solve");
    CK(cudaSetDevice(ctx->device));
    if (ctx->running) {
        int32_t busy = 0;
        CK(cudaEventSynchronize(ctx->ev[1]));
        int rc0 = prt_ctx_busy(ctx, &busy);
        if (rc0 != PRT_OK) return rc0;
    }
    FlowState& F = ctx->flow;
    FlowCtrl res;
    CK(cudaMemcpyAsync(&res, F.ctrl.p, sizeof(res), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (!res.done) return fail(ctx, PRT_E_STATE, "the flow loop has not finished");
    int rc = flow_finish(ctx, info);
    if (rc != PRT_OK) return rc;
    ctx->flow_armed = false;
    ctx->timing[1] = (double)res.iters;
    if (vel_out) {
        CK(cudaMemcpyAsync(vel_out, F.d_vel, (size_t)F.g.n * 3 * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return PRT_OK;
}

extern "C" int prt_adr_stage_flow(prt_ctx* ctx, const prt_adr_geom* geom, prt_adr_stats* stats) {
    if (!ctx || !geom) return fail(ctx, PRT_E_INVALID, "null argument");
    if (ctx->batch) return fail(ctx, PRT_E_STATE, "the context is in a batch");
    FlowState& F = ctx->flow;
    if (!F.field_ready || !F.d_mat || !F.d_vel)
        return fail(ctx, PRT_E_STATE, "no finished flow field on this context");
    const Grid g = make_grid(geom->nd, geom->dims);
    if (geom->nd != F.p.nd || g.n != F.g.n || g.nx != F.g.nx || g.ny != F.g.ny || g.nz != F.g.nz)
        return fail(ctx, PRT_E_INVALID, "the transport grid differs from the flow grid");
    return prt_adr_stage_dev(ctx, F.d_mat, F.d_vel, geom, stats);
}

extern "C" int prt_flow_release(prt_ctx* ctx) {
    if (!ctx) return PRT_E_INVALID;
    // a context in a batch may drop its lattices once its flow solve is
    // finished: the batch's kernels no longer touch them
    if (ctx->batch && ctx->flow_armed)
        return fail(ctx, PRT_E_STATE, "the context's flow solve is in a batch");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->flow.release_lattices();
    ctx->flow_armed = false;
    return PRT_OK;
}

extern "C" int prt_adr_start(prt_ctx* ctx, const prt_adr_run_params* rp) {
    if (!ctx || !rp) return fail(ctx, PRT_E_INVALID, "null argument");
    if (ctx->batch) return fail(ctx, PRT_E_STATE, "the context is in a batch");
    if (ctx->flow_armed) return fail(ctx, PRT_E_STATE, "the context's flow solve is unfinished");
    ctx->adr_armed = false;
    int rc = adr_run_setup(ctx, rp, rp->limit);  // synchronises its stream
    if (rc != PRT_OK) return rc;
    ctx->adr_armed = true;
    return PRT_OK;
}

extern "C" int prt_adr_finish(prt_ctx* ctx, prt_adr_result* res) {
    if (!ctx) return PRT_E_INVALID;
    if (ctx->batch) return fail(ctx, PRT_E_STATE, "the context is in a batch");
    if (!ctx->adr_armed) return fail(ctx, PRT_E_STATE, "no started transport run");
    CK(cudaSetDevice(ctx->device));
    if (ctx->running) {
        int32_t busy = 0;
        CK(cudaEventSynchronize(ctx->ev[3]));
        int rc0 = prt_ctx_busy(ctx, &busy);
        if (rc0 != PRT_OK) return rc0;
    }
    AdrCtrl cur;
    CK(cudaMemcpyAsync(&cur, ctx->adr.ctrl.p, sizeof(cur), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (!cur.done) return fail(ctx, PRT_E_STATE, "the transport loop has not finished");
    int rc = adr_run_finish(ctx, res);
    if (rc != PRT_OK) return rc;
    ctx->adr_armed = false;
    ctx->timing[3] = (double)cur.n_base;
    return PRT_OK;
}

// ===========================================================================
// concurrent solves: each loop enqueued on its context's own stream
// ===========================================================================
extern "C" int prt_flow_launch(prt_ctx* ctx) {
    if (!ctx) return PRT_E_INVALID;
    if (ctx->batch) return fail(ctx, PRT_E_STATE, "the context is in a batch");
    if (!ctx->flow_armed) return fail(ctx, PRT_E_STATE, "no started flow solve");
    if (ctx->running) return fail(ctx, PRT_E_STATE, "a loop is already running on this context");
    CK(cudaSetDevice(ctx->device));
    int rc = flow_loop_async(ctx);
    if (rc != PRT_OK) return rc;
    ctx->running = 1;
    return PRT_OK;
}

extern "C" int prt_adr_launch(prt_ctx* ctx) {
    if (!ctx) return PRT_E_INVALID;
    if (ctx->batch) return fail(ctx, PRT_E_STATE, "the context is in a batch");
    if (!ctx->adr_armed) return fail(ctx, PRT_E_STATE, "no started transport run");
    if (ctx->running) return fail(ctx, PRT_E_STATE, "a loop is already running on this context");
    CK(cudaSetDevice(ctx->device));
    int rc = adr_loop_async(ctx);
    if (rc != PRT_OK) return rc;
    ctx->running = 2;
    return PRT_OK;
}

extern "C" int prt_ctx_busy(prt_ctx* ctx, int32_t* busy) {
    if (!ctx || !busy) return PRT_E_INVALID;
    *busy = 0;
    if (!ctx->running) return PRT_OK;
    CK(cudaSetDevice(ctx->device));
    cudaEvent_t a = ctx->running == 1 ? ctx->ev[0] : ctx->ev[2];
    cudaEvent_t b = ctx->running == 1 ? ctx->ev[1] : ctx->ev[3];
    const cudaError_t e = cudaEventQuery(b);
    if (e == cudaErrorNotReady) {
        *busy = 1;
        return PRT_OK;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaEventQuery");
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    ctx->timing[ctx->running == 1 ? 0 : 2] = ms;
    ctx->running = 0;
    return PRT_OK;
}

// ===========================================================================
// batch
// ===========================================================================
extern "C" int prt_batch_create(int device, int32_t graph_steps, prt_batch** out) {
    if (!out) return PRT_E_INVALID;
    *out = nullptr;
    if (graph_steps < 0 || graph_steps > 4096) return PRT_E_INVALID;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_noctx_error("no CUDA device");
        return PRT_E_NODEV;
    }
    if (device < 0 || device >= n) return PRT_E_INVALID;
    prt_batch* b = new (std::nothrow) prt_batch();
    if (!b) return PRT_E_OOM;
    b->device = device;
    b->K = graph_steps ? graph_steps : 20;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&b->t0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->t1);
    if (e == cudaSuccess) e = b->d_gstep.fit(sizeof(long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_gstep.b.p, 0, sizeof(long long), b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        set_noctx_error(cudaGetErrorString(e));
        prt_batch_destroy(b);
        return PRT_E_CUDA;
    }
    *out = b;
    return PRT_OK;
}

extern "C" void prt_batch_destroy(prt_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    {
        std::lock_guard<std::mutex> lk(b->mu);
        for (prt_ctx* c : b->jobs) c->batch = nullptr;
        b->jobs.clear();
    }
    b->graph.release();
    GrowBuf* all[] = {&b->d_flow, &b->d_adr, &b->d_done, &b->d_status, &b->d_arrive,
                      &b->d_adr_cnt, &b->d_counts, &b->d_gstep};
    for (GrowBuf* g : all) g->b.release();
    for (int c = 0; c < kClasses; ++c) b->d_tiles[c].b.release();
    if (b->h_status) cudaFreeHost(b->h_status);
    cudaEvent_t evs[] = {b->fork, b->t0, b->t1};
    for (cudaEvent_t ev : evs)
        if (ev) cudaEventDestroy(ev);
    for (int c = 0; c < kClasses; ++c) {
        if (b->cls_join[c]) cudaEventDestroy(b->cls_join[c]);
        if (b->cls_stream[c]) cudaStreamDestroy(b->cls_stream[c]);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

extern "C" const char* prt_batch_last_error(const prt_batch* b) { return b ? b->err.c_str() : ""; }

extern "C" int prt_batch_add(prt_batch* b, prt_ctx* job) {
    if (!b || !job) return bfail(b, PRT_E_INVALID, "null argument");
    if (job->batch) return bfail(b, PRT_E_STATE, "the context is already in a batch");
    if (job->device != b->device) return bfail(b, PRT_E_INVALID, "the context is on another device");
    if (!job->flow_armed && !job->adr_armed)
        return bfail(b, PRT_E_STATE, "the context has no started flow solve or transport run");
    if (job->running) return bfail(b, PRT_E_STATE, "the context's loop is running on its stream");
    // the count the job joins with (the batch advances it implicitly)
    BK(cudaSetDevice(job->device));
    long long c0 = 0;
    const char* src = job->flow_armed
                          ? job->flow.ctrl.as<const char>() + offsetof(FlowCtrl, it_base)
                          : job->adr.ctrl.as<const char>() + offsetof(AdrCtrl, n_base);
    BK(cudaMemcpyAsync(&c0, src, sizeof(c0), cudaMemcpyDeviceToHost, job->stream));
    BK(cudaStreamSynchronize(job->stream));
    std::lock_guard<std::mutex> lk(b->mu);
    b->jobs.push_back(job);
    job->batch = b;
    job->batch_c0 = c0;
    job->batch_g0_set = false;
    b->dirty = true;
    return PRT_OK;
}

extern "C" int prt_batch_remove(prt_batch* b, prt_ctx* job) {
    if (!b || !job) return bfail(b, PRT_E_INVALID, "null argument");
    if (job->batch != b) return bfail(b, PRT_E_INVALID, "the context is not in this batch");
    if (b->in_flight) return bfail(b, PRT_E_STATE, "wait for the launch before removing jobs");
    // a job leaving before its loop ended gets its count written back: the
    // batch writes it to the control block only on the steps that check
    if (job->batch_g0_set) {
        BK(cudaSetDevice(b->device));
        const long long count = b->steps_run - job->batch_g0;
        cudaStream_t s = job->stream;
        if (job->flow_armed) {
            FlowCtrl fc;
            BK(cudaMemcpyAsync(&fc, job->flow.ctrl.p, sizeof(fc), cudaMemcpyDeviceToHost, s));
            BK(cudaStreamSynchronize(s));
            if (!fc.done) {
                fc.it_base = count;
                fc.iters = count;
                BK(cudaMemcpyAsync(job->flow.ctrl.p, &fc, sizeof(fc), cudaMemcpyHostToDevice, s));
                BK(cudaStreamSynchronize(s));
            }
        } else {
            AdrCtrl ac;
            BK(cudaMemcpyAsync(&ac, job->adr.ctrl.p, sizeof(ac), cudaMemcpyDeviceToHost, s));
            BK(cudaStreamSynchronize(s));
            if (!ac.done) {
                ac.n_base = count;
                BK(cudaMemcpyAsync(job->adr.ctrl.p, &ac, sizeof(ac), cudaMemcpyHostToDevice, s));
                BK(cudaStreamSynchronize(s));
            }
        }
    }
    batch_detach(job);
    return PRT_OK;
}

extern "C" int prt_batch_launch(prt_batch* b, int32_t steps) {
    if (!b) return PRT_E_INVALID;
    if (steps < 0) return bfail(b, PRT_E_INVALID, "negative step count");
    if (b->in_flight) return bfail(b, PRT_E_STATE, "the previous launch was not waited for");
    BK(cudaSetDevice(b->device));
    std::lock_guard<std::mutex> lk(b->mu);
    if (b->dirty && b->auto_tile && !b->tuning && !b->jobs.empty()) {
        long long blocks = 0;
        const double share = flow_share(b, &blocks);
        if (std::fabs(share - b->tune_share) > kRetuneShift ||
            (double)blocks * kRetuneScale < (double)b->tune_blocks ||
            (double)blocks > kRetuneScale * (double)b->tune_blocks) {
            b->tuning = true;
            b->cand = 0;
            b->cand_pass = 0;
        }
    }
    if (b->tuning && b->cand == 0 && b->cand_pass == 0)
        b->tune_share = flow_share(b, &b->tune_blocks);
    if (b->tuning) {
        const Candidate& cd = kCandidates[b->cand];
        if (cd.tile_blocks != b->tile_blocks || cd.grid_mult != b->grid_mult) {
            b->tile_blocks = cd.tile_blocks;
            b->grid_mult = cd.grid_mult;
            b->dirty = true;
        }
    }
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc != PRT_OK) return rc;
    }
    const int njobs = (int)b->order.size();
    const int replays = (steps + b->K - 1) / b->K;
    cudaStream_t s = b->stream;
    const bool use_graph = !graphs_disabled();
    if (njobs > 0 && replays > 0 && use_graph) {
        int rc = ensure_graph(b);
        if (rc != PRT_OK) return rc;
    }
    BK(cudaEventRecord(b->t0, s));
    if (njobs > 0 && replays > 0) {
        if (!use_graph) {
            for (int r = 0; r < replays; ++r) {
                // without a graph every class goes on the batch stream
                for (int k = 0; k < b->K; ++k) {
                    cudaError_t e = emit_step(b, s, nullptr, k);
                    if (e != cudaSuccess) return bcuda(b, e, "batch step launch");
                }
                BK(batch_launch_gstep(b->d_gstep.b.as<long long>(), b->K, s));
            }
        } else {
            for (int r = 0; r < replays; ++r) BK(cudaGraphLaunch(b->graph.exec, s));
        }
        b->launches += (int64_t)replays * (b->K * launches_per_step(b) + 1);
    }
    if (njobs > 0) {
        BK(batch_launch_status(b->d_done.b.as<const int* const>(), njobs, b->d_status.b.as<int>(), s));
        BK(cudaMemcpyAsync(b->h_status, b->d_status.b.p, (size_t)njobs * sizeof(int),
                           cudaMemcpyDeviceToHost, s));
        b->launches += 1;
    }
    BK(cudaEventRecord(b->t1, s));
    b->in_flight = true;
    b->launch_replays = (njobs > 0) ? replays : 0;
    b->steps_run += (int64_t)b->launch_replays * b->K;
    return PRT_OK;
}

extern "C" int prt_batch_wait(prt_batch* b, int32_t* n_done) {
    if (!b) return PRT_E_INVALID;
    if (!b->in_flight) {
        if (n_done) *n_done = 0;
        return PRT_OK;
    }
    BK(cudaSetDevice(b->device));
    b->in_flight = false;
    BK(cudaEventSynchronize(b->t1));
    float ms = 0.f;
    BK(cudaEventElapsedTime(&ms, b->t0, b->t1));
    b->last_ms = ms;
    std::lock_guard<std::mutex> lk(b->mu);
    int done = 0;
    for (size_t i = 0; i < b->order.size(); ++i)
        if (b->order[i] && b->h_status[i]) ++done;
    if (n_done) *n_done = done;
    // tiling choice: cost per block-step of each candidate, then the cheapest
    if (b->tuning && b->launch_replays > 0 && b->launch_blocks > 0) {
        const double cost = ms / ((double)b->launch_replays * b->K * (double)b->launch_blocks);
        if (b->cand_pass == 0 || cost < b->cand_cost[b->cand]) b->cand_cost[b->cand] = cost;
        if (++b->cand_pass == kTunePasses) {
            b->cand_pass = 0;
            b->cand += 1;
        }
        if (b->cand == kNumCandidates) {
            int best = 0;
            for (int i = 1; i < kNumCandidates; ++i)
                if (b->cand_cost[i] < b->cand_cost[best]) best = i;
            b->tuning = false;
            if (kCandidates[best].tile_blocks != b->tile_blocks ||
                kCandidates[best].grid_mult != b->grid_mult) {
                b->tile_blocks = kCandidates[best].tile_blocks;
                b->grid_mult = kCandidates[best].grid_mult;
                b->dirty = true;
            }
        }
    }
    return PRT_OK;
}

extern "C" int prt_batch_run(prt_batch* b, int32_t steps, int32_t* n_done) {
    int rc = prt_batch_launch(b, steps);
    if (rc != PRT_OK) return rc;
    return prt_batch_wait(b, n_done);
}

extern "C" int prt_batch_collect(prt_batch* b, prt_ctx** out, int32_t cap, int32_t* count) {
    if (!b) return PRT_E_INVALID;
    if (b->in_flight) return bfail(b, PRT_E_STATE, "wait for the launch before collecting");
    int n = 0;
    std::vector<prt_ctx*> done;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        for (size_t i = 0; i < b->order.size() && n < cap; ++i) {
            prt_ctx* c = b->order[i];
            if (!c || !b->h_status[i]) continue;
            if (out) out[n] = c;
            ++n;
            done.push_back(c);
            b->order[i] = nullptr;
        }
    }
    for (prt_ctx* c : done) batch_detach(c);
    if (count) *count = n;
    return PRT_OK;
}

extern "C" int prt_batch_size(const prt_batch* b, int32_t* flow_jobs, int32_t* adr_jobs) {
    if (!b) return PRT_E_INVALID;
    prt_batch* m = const_cast<prt_batch*>(b);
    std::lock_guard<std::mutex> lk(m->mu);
    int nf = 0, na = 0;
    for (prt_ctx* c : b->jobs) (is_flow_job(c) ? nf : na) += 1;
    if (flow_jobs) *flow_jobs = nf;
    if (adr_jobs) *adr_jobs = na;
    return PRT_OK;
}

extern "C" int prt_batch_tune(prt_batch* b, int32_t tile_blocks, int32_t grid_mult) {
    if (!b) return PRT_E_INVALID;
    std::lock_guard<std::mutex> lk(b->mu);
    if (tile_blocks == 0) {
        b->auto_tile = true;
        b->tuning = true;
        b->cand = 0;
        b->cand_pass = 0;
        return PRT_OK;
    }
    if (!(tile_blocks == 1 || tile_blocks == 2 || tile_blocks == 4) ||
        !(grid_mult == 0 || grid_mult == 1 || grid_mult == 2))
        return bfail(b, PRT_E_INVALID,
                     "tile blocks must be 1, 2 or 4 and the grid multiple 0, 1 or 2");
    b->auto_tile = false;
    b->tuning = false;
    if (tile_blocks != b->tile_blocks || grid_mult != b->grid_mult) b->dirty = true;
    b->tile_blocks = tile_blocks;
    b->grid_mult = grid_mult;
    return PRT_OK;
}

extern "C" int prt_batch_stats(const prt_batch* b, double* out8) {
    if (!b || !out8) return PRT_E_INVALID;
    out8[0] = (double)b->launches;
    out8[1] = (double)b->graph_builds;
    out8[2] = b->tile_blocks;
    out8[3] = b->grid_mult;
    out8[4] = (double)b->steps_run;
    out8[5] = b->last_ms;
    out8[6] = (double)b->last_tiles;
    out8[7] = b->tuning ? 1.0 : 0.0;
    return PRT_OK;
}

extern "C" int prt_mem_info(int device, uint64_t* free_bytes, uint64_t* total_bytes) {
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        set_noctx_error("no CUDA device");
        return PRT_E_NODEV;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        set_noctx_error("device index out of range");
        return PRT_E_INVALID;
    }
    size_t fr = 0, to = 0;
    cudaError_t e = cudaMemGetInfo(&fr, &to);
    cudaSetDevice(cur);
    if (e != cudaSuccess) {
        set_noctx_error(cudaGetErrorString(e));
        return PRT_E_CUDA;
    }
    if (free_bytes) *free_bytes = fr;
    if (total_bytes) *total_bytes = to;
    return PRT_OK;
}
