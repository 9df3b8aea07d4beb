// runtime_internal.h -- host-side state of a context (prt_ctx) and the
// helpers shared by runtime.cu (single solves) and engine.cu (batches).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "prt_internal.h"

namespace prt {
cudaError_t adr_launch_chunk_means(const AdrDev& d, AdrCtrl* ctrl, const float** src_slot,
                                   float* means_out, cudaStream_t s);
cudaError_t adr_launch_flags(const uint8_t* mat, const Grid& g, int nd, int pore, int bfc,
                             uint32_t* flags, uint8_t* mflag, cudaStream_t s);
cudaError_t adr_launch_vel_stats(const float* vel, const AdrDev& d, float* tmp, float* means,
                                 unsigned* vmax_bits, unsigned long long* nbf, cudaStream_t s);

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t want) {
        if (want <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, want ? want : 1);
        if (e == cudaSuccess) bytes = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct GraphHolder {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool conditional = false;
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

struct FlowKey {
    int nd = 0, precision = -1, every = 0;
    Grid g{0, 0, 0, 0};
    double force = 0, tau = 0, magic = 0;
    long long nit = -1;
    double tol = 0;
    void* f = nullptr;
    void* aux[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    long long nf = -1;  // pore voxels: launch sizes and the lattice stride are baked in
    int pdl = 0;        // the launch settings the step kernels were captured with (pdl_key)
    bool operator==(const FlowKey& o) const {
        return nd == o.nd && precision == o.precision && every == o.every && g.nx == o.g.nx &&
               g.ny == o.g.ny && g.nz == o.g.nz && force == o.force && tau == o.tau &&
               magic == o.magic && nit == o.nit && tol == o.tol && f == o.f && aux[0] == o.aux[0] &&
               aux[1] == o.aux[1] && aux[2] == o.aux[2] && aux[3] == o.aux[3] &&
               aux[4] == o.aux[4] && nf == o.nf && pdl == o.pdl;
    }
};

struct FlowState {
    DevBuf f, fluid, partials, ctrl, out5, count, mat, vel, flag, cnt, cells, nbr;
    GraphHolder graph;
    FlowKey key;
    // the solve set up by flow_setup
    prt_flow_params p{};
    Grid g{0, 0, 0, 0};
    FlowMap fm{0, nullptr, nullptr, 0, 0, nullptr};
    LbParams kc{};
    int nb = 1;
    long long nfluid = 0;
    float scale = 1.f;
    const uint8_t* d_mat = nullptr;  // material grid of the solve (borrowed)
    float* d_vel = nullptr;          // its output field (borrowed)
    bool field_ready = false;        // d_vel holds the final field
    void release_lattices() {
        DevBuf* all[] = {&f, &fluid, &partials, &count, &flag, &cnt, &cells, &nbr};
        for (DevBuf* b : all) b->release();
        graph.release();
        key = FlowKey();
    }
};

struct AdrState {
    bool begun = false;
    bool ran = false;
    prt_adr_params p{};
    AdrDev d{};
    DevBuf mat, vel, flags, mflag, face[3], buf[2], ladder, slot_of_step, idx, cnt, total;
    DevBuf tree_leaf_start, tree_leaf_len, tree_inner_l, tree_inner_r, tree_level_off, tree_vals;
    DevBuf means, src_slot, ctrl, log;
    // for the batch engine: blk_leaf[b] = the first leaf starting at or after
    // solute voxel kBatchAdrBlock * b (b = 0 .. nbk), see AdrJob
    DevBuf blk_leaf;
    int nbk = 0;
    bool staged = false;
    prt_adr_geom geom{};
    const uint8_t* d_mat = nullptr;  // staged inputs (borrowed until begin)
    const float* d_vel = nullptr;
    DevBuf tmp, vstats;
    std::vector<long long> sched;       // ladder step schedule of the run
    prt_adr_run_params rp{};
    std::vector<long long> keep_steps;  // ladder step numbers
    std::vector<int> slot_of_index;     // ladder index -> slot
    int nslots = 0;
    GraphHolder graph;
    // what the loop graph bakes in (adr_graph_key): a run whose key equals
    // the cached graph's replays it instead of capturing a new one
    std::vector<unsigned char> graph_key;
    // Ends the transport state.  Device buffers of at most keep_bytes stay
    // with the context for its next run (every run sizes them with ensure()
    // and initialises what it reads), so back-to-back solves on one context
    // do not pay cudaFree / cudaMalloc each time; larger ones are freed.
    void release(size_t keep_bytes = 0) {
        DevBuf* all[] = {&mat, &vel, &flags, &mflag, &face[0], &face[1], &face[2], &buf[0], &buf[1],
                         &ladder, &slot_of_step, &idx, &cnt, &total, &tree_leaf_start,
                         &tree_leaf_len, &tree_inner_l, &tree_inner_r, &tree_level_off, &tree_vals,
                         &means, &src_slot, &ctrl, &log, &tmp, &vstats, &blk_leaf};
        bool freed = false;
        for (DevBuf* b : all)
            if (b->bytes > keep_bytes) {
                freed = freed || b->p != nullptr;
                b->release();
            }
        staged = false;
        // the cached loop graph holds device pointers: it goes with any
        // buffer that is freed (a kept run's next key compares them anyway)
        if (freed || keep_bytes == 0) {
            graph.release();
            graph_key.clear();
        }
        keep_steps.clear();
        slot_of_index.clear();
        begun = ran = false;
    }
};

// Device buffers of the inlet walk (prep.cu) and of the check_physics
// reductions (physics.cu), kept for the next call.
struct PrepState {
    DevBuf mat, steps, flags, counts, keys, sums, out;
    long long staged_out = -1;  // floats of the staged check_physics result (-1: none)
    long long staged_mat = -1;  // voxels of the staged material grid
    void release() {
        DevBuf* all[] = {&mat, &steps, &flags, &counts, &keys, &sums, &out};
        staged_out = staged_mat = -1;
        for (DevBuf* b : all) b->release();
    }
};

}  // namespace prt

struct prt_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int64_t launches = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double timing[4] = {0, 0, 0, 0};
    prt::FlowState flow;
    prt::AdrState adr;
    prt::PrepState prep;
    bool flow_armed = false;  // flow set up, its time loop not finished
    bool adr_armed = false;   // transport run set up, its time loop not finished
    prt_batch* batch = nullptr;  // the batch holding this context, if any
    long long batch_c0 = 0;      // iterations / steps done when it joined the batch
    long long batch_g0 = 0;      // its count is (batch steps done) - batch_g0
    bool batch_g0_set = false;   // batch_g0 is fixed at the first launch after joining
    int running = 0;             // a loop enqueued by prt_*_launch: 1 flow, 2 transport
    long long l2_bytes = 0;      // the device's L2 cache
};

namespace prt {

inline int fail(prt_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

inline int cuda_fail(prt_ctx* c, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(c, e == cudaErrorMemoryAllocation ? PRT_E_OOM : PRT_E_CUDA, m);
}

#define CK(expr)                                                   \
    do {                                                           \
        cudaError_t _e = (expr);                                   \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #expr);   \
    } while (0)

inline bool graphs_disabled() {
    const char* v = std::getenv("PRT_GRAPHS");
    return v && v[0] == '0';
}

// Build "while (cond) { body }" as a graph; body is captured from `emit`.
// Falls back to a plain graph of the body when conditional nodes are
// unavailable (the host then relaunches it until the control block says done).
template <class Emit>
inline cudaError_t build_while_graph(cudaStream_t s, GraphHolder& gh, Emit emit) {
    gh.release();
    cudaError_t e = cudaGraphCreate(&gh.graph, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle handle;
    e = cudaGraphConditionalHandleCreate(&handle, gh.graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        e = cudaGraphAddNode(&node, gh.graph, nullptr, 0, &cp);
        if (e == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t ee = emit(handle, 1);
                cudaGraph_t outg = nullptr;
                e = cudaStreamEndCapture(s, &outg);
                if (ee != cudaSuccess) e = ee;
                if (e == cudaSuccess) {
                    e = cudaGraphInstantiate(&gh.exec, gh.graph, 0);
                    if (e == cudaSuccess) {
                        gh.conditional = true;
                        return cudaSuccess;
                    }
                }
            }
        }
    }
    // fallback: plain body graph
    cudaGetLastError();
    gh.release();
    e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t ee = emit(cudaGraphConditionalHandle(0), 0);
    e = cudaStreamEndCapture(s, &gh.graph);
    if (ee != cudaSuccess) return ee;
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&gh.exec, gh.graph, 0);
    gh.conditional = false;
    return e;
}

inline Grid make_grid(int nd, const int32_t* dims) {
    Grid g;
    if (nd == 3) {
        g.nx = dims[0];
        g.ny = dims[1];
        g.nz = dims[2];
    } else {
        g.nx = dims[0];
        g.ny = 1;
        g.nz = dims[1];
    }
    g.n = (long long)g.nx * g.ny * g.nz;
    return g;
}


// The three parts of a single solve, also driven by the batch engine:
// set-up, the time loop (single or batched), the results.
int flow_setup(prt_ctx* ctx, const uint8_t* d_mat, const prt_flow_params* p, float* d_vel);
int flow_finish(prt_ctx* ctx, prt_flow_info* info);
int adr_run_setup(prt_ctx* ctx, const prt_adr_run_params* rp, long long pause_every);
int adr_run_finish(prt_ctx* ctx, prt_adr_result* res);
// Enqueue the whole flow / transport loop of a started solve on the
// context's stream without waiting (runtime.cu).
int flow_loop_async(prt_ctx* ctx);
int adr_loop_async(prt_ctx* ctx);
// Takes ctx out of its batch (engine.cu); used by prt_destroy.
void batch_detach(prt_ctx* ctx);

}  // namespace prt
