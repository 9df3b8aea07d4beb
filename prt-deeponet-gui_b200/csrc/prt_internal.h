// prt_internal.h -- structures shared by the kernel translation units and the
// host runtime of libprtlb.so.  Not part of the public ABI (include/prtlb.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdlib>

#include "../../include/prtlb.h"

namespace prt {

// A grid in the storage frame.  3D (nx, ny, nz) is kept as is; a 2D (nx, ny)
// grid is stored as (nx, 1, ny) so that the contiguous axis is always the
// last one and the linear index (x*ny + y) is unchanged.
struct Grid {
    int nx, ny, nz;
    long long n;  // nx*ny*nz
};

// Division by a divisor fixed for a whole run as one high multiply, one add
// and one shift: the round-up method of Granlund and Montgomery ("Division
// by invariant integers using multiplication", PLDI 1994) with a 33-bit
// multiplier 2^32 + m, s = ceil(log2 d).  Exact for 0 <= t < 2^31 (then
// the add cannot carry out of 32 bits).
struct FastDiv {
    unsigned d, m;
    int s;
};

inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d;
    f.s = 0;
    while (f.s < 31 && (1u << f.s) < d) ++f.s;
    const unsigned long long two32 = 1ull << 32;
    f.m = (unsigned)((two32 * ((1ull << f.s) - d)) / d + 1);
    return f;
}

#ifdef __CUDACC__
__device__ __forceinline__ unsigned fast_div(unsigned t, const FastDiv& f) {
    return (__umulhi(t, f.m) + t) >> f.s;
}
#endif

#ifdef __CUDACC__
// Programmatic dependent launch: let the next kernel in the stream start
// launching now, and wait until the previous one has finished and its
// stores are visible (both no-ops for a kernel launched without the
// programmatic-serialisation attribute).
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" :::);
}
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
#endif

// Whether step launches (flow, batched flow, transport) carry the
// programmatic-serialisation attribute; PRT_PDL=0 launches them plainly.
inline bool pdl_enabled() {
    const char* v = std::getenv("PRT_PDL");
    return !(v && v[0] == '0');
}

// Where a single-solve step kernel lets the next step launch
// (griddepcontrol.launch_dependents): after its own stores when its grid
// fits in one resident wave -- the next step's blocks then arrive as this
// one drains instead of sitting beside it (64^3: flow 4.60 -> 4.09 us per
// iteration, transport 4.11 -> 3.66 us per step) -- and at its start when
// it does not, so later waves overlap the next step's set-up.
// PRT_PDL_LATE=all / none puts it at the end / the start for every grid.
inline bool pdl_late(bool one_wave) {
    const char* v = std::getenv("PRT_PDL_LATE");
    if (v && v[0] == 'a') return true;
    if (v && v[0] == 'n') return false;
    return one_wave;
}

// The launch settings a captured loop graph bakes in (PRT_PDL, PRT_PDL_LATE),
// as one number for the graph caches' keys.
inline int pdl_key() {
    const char* v = std::getenv("PRT_PDL_LATE");
    const int late = (v && v[0] == 'a') ? 1 : (v && v[0] == 'n') ? 2 : 0;
    return (pdl_enabled() ? 1 : 0) + 2 * late;
}

// Device-side state of FlowConvergence (prtlb_3d.py:168-252) for one solve.
struct FlowCtrl {
    long long it_base;  // iterations completed before the current chunk
    long long nit;      // cap
    long long iters;    // flow_iters
    long long nfluid;
    double tol;
    double prev;
    double change;
    int every;
    int done;
    int has_prev;
    int converged;
    int nonfinite;  // sticky: a sampled mean |u_x| was NaN or infinite
    int pad;
};

// Constants of one flow solve, in float64; kernels round them to their
// arithmetic type.
struct LbParams {
    double omp, omm;  // omega+ , omega-
    double half_g;    // force / 2, added to the x momentum
    double guo[9];    // w_a (1 - omega-/2) 3 g c_ax for the first member of each pair
    float scale;      // FP16 storage scale (2^k) and its inverse
    float inv_scale;
};

// Control block of one transport solve (the while loop of prtlb_3d.py:1493).
struct AdrCtrl {
    long long n_base;  // steps completed before the current chunk
    long long limit;
    long long n_pause;  // host asked to regain control at this step
    long long checks;
    int check;
    int until_conv;
    int done;
    int converged;
    int ns;
    int nlog;
    double tol;
    double last_rest;
    double prev[PRT_MAX_SPECIES];
    double prev_change[PRT_MAX_SPECIES];
    double scale[PRT_MAX_SPECIES];
};

struct ProgressRec {
    long long n;
    double mean0;
    double value;
};

// Flag bits of one transport voxel (built once per solve by adr_setup).
enum : uint32_t {
    F_M = 1u << 0,        // solute voxel (pore or biofilm)
    F_BF = 1u << 1,       // biofilm voxel
    F_X0 = 1u << 2,       // on the x = 0 face (the inlet plane)
    // per axis a (0..2): open_lo, open_hi, far_lo, far_hi at 3 + 4a
    F_AX0 = 3,
    // biofilm neighbour lo/hi per axis a at 15 + 2a
    F_NBF0 = 15,
};

__host__ __device__ inline uint32_t f_open_lo(int a) { return 1u << (F_AX0 + 4 * a + 0); }
__host__ __device__ inline uint32_t f_open_hi(int a) { return 1u << (F_AX0 + 4 * a + 1); }
__host__ __device__ inline uint32_t f_far_lo(int a) { return 1u << (F_AX0 + 4 * a + 2); }
__host__ __device__ inline uint32_t f_far_hi(int a) { return 1u << (F_AX0 + 4 * a + 3); }
__host__ __device__ inline uint32_t f_nbf_lo(int a) { return 1u << (F_NBF0 + 2 * a + 0); }
__host__ __device__ inline uint32_t f_nbf_hi(int a) { return 1u << (F_NBF0 + 2 * a + 1); }

// numpy's float32 pairwise summation tree over the solute voxels, flattened:
// leaves [0, nleaf) sum runs of <= 128 consecutive compressed values, internal
// nodes [nleaf, nleaf + ninner) add two earlier values; inner nodes are sorted
// by height so each height is one parallel level.
struct PairTree {
    int nleaf;
    int ninner;
    int nlevel;
    int root;             // value index of the root (-1 when there are no voxels)
    const int* leaf_start;
    const int* leaf_len;
    const int* inner_l;
    const int* inner_r;
    const int* level_off;  // nlevel + 1 offsets into the inner arrays
};

// The pore-only layout of a flow solve: lattice slot k holds the k-th pore
// voxel in C order, whose coordinates are packed in cells[k] as
// x << xs | y << ys | z (so a kernel finds its neighbours with shifts and
// masks instead of divisions); imap[voxel] is the slot of a pore voxel, -1
// for rock.  nbr, when not null, holds the pull tables, one per parity p of
// the read lattice: nbr[p * (Q-1) * nf + (i - 1) * nf + k] = the element
// offset (into the two lattices) slot k pulls direction i from -- the
// upstream slot of the read lattice, or slot k's own opp(i) of the write
// lattice when that voxel is rock (i = 1 .. Q-1).  The step kernel then
// reads them in one coalesced pass instead of the packed cell, the imap
// lookups and the choice between the two lattices.  Set up for solves whose
// lattices and tables fit in half the L2 cache, where the latency of the
// lookups, not the bytes of the tables, bounds an iteration.
struct FlowMap {
    int nf;
    const int* cells;
    const int* imap;
    int ys, xs;  // bit offsets of y and x in a packed cell
    const int* nbr;
};

// Bytes of the two pull tables of nf pore voxels (Q-1 ints each per parity).
inline long long flow_nbr_bytes(int q, long long nf) { return 2ll * (q - 1) * nf * 4; }

// Whether a solve with nf pore voxels and populations of es bytes gets the
// pull tables on a device with l2_bytes of L2: when the two lattices and one
// table (an iteration reads one) fit in half of it.
inline bool flow_use_nbr(int q, long long nf, long long es, long long l2_bytes) {
    return nf > 0 && 2 * q * nf * es + flow_nbr_bytes(q, nf) / 2 <= l2_bytes / 2;
}

// Constants of one flow solve (the TRT rates of _trt_minus and the Guo
// force terms), shared by every entry point that runs a flow solve.
inline void fill_lbconst(LbParams& k, int nd, double force, double tau, double magic, float scale) {
    // _trt_minus (prtlb_3d.py:130-139)
    const double om_p = 1.0 / tau;
    const double lam_p = 1.0 / om_p - 0.5;
    const double om_m = 1.0 / (magic / lam_p + 0.5);
    k.omp = om_p;
    k.omm = om_m;
    k.half_g = 0.5 * force;
    for (int p = 0; p < 9; ++p) k.guo[p] = 0.0;
    // first member of each pair and its x component
    if (nd == 3) {
        // pairs (1,2) (3,4) ... (17,18); e_x of 1,7,9,11,13 is +1, of 3,5,15,17 is 0
        const int pa[9] = {1, 3, 5, 7, 9, 11, 13, 15, 17};
        const int ex[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
        for (int p = 0; p < 9; ++p) {
            const int a = pa[p];
            const double w = a < 7 ? 1.0 / 18.0 : 1.0 / 36.0;
            k.guo[p] = w * (1 - 0.5 * om_m) * 3.0 * force * ex[a];
        }
    } else {
        const int pa[4] = {1, 2, 5, 6};
        const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
        for (int p = 0; p < 4; ++p) {
            const int a = pa[p];
            const double w = a < 5 ? 1.0 / 9.0 : 1.0 / 36.0;
            k.guo[p] = w * (1 - 0.5 * om_m) * 3.0 * force * ex[a];
        }
    }
    k.scale = scale;
    k.inv_scale = 1.0f / scale;
}

// Bits that hold the values 0 .. n-1.
__host__ __device__ inline int coord_bits(int n) {
    int b = 0;
    while (b < 31 && (1 << b) < n) ++b;
    return b;
}

__host__ __device__ inline void unpack_cell(unsigned cv, const FlowMap& fm, int& x, int& y,
                                            int& z) {
    z = (int)(cv & ((1u << fm.ys) - 1u));
    y = (int)((cv >> fm.ys) & ((1u << (fm.xs - fm.ys)) - 1u));
    x = (int)(cv >> fm.xs);
}

// Kernel launchers (lb_flow.cu) ---------------------------------------------
// Returns cudaSuccess or the launch error.  f holds the two lattices (read /
// write swap with the iteration parity), Q * nf populations each.  Step and
// moments launches have flow_blocks(nf) blocks (the partial-sum count).
cudaError_t flow_launch_step(int nd, int precision, bool odd, bool check, void* f,
                             const FlowMap& fm, const Grid& g, const LbParams& lbp,
                             const FlowCtrl* ctrl, int kstep, double* partials,
                             cudaStream_t s);
cudaError_t flow_launch_check(FlowCtrl* ctrl, const double* partials, int nblocks,
                              cudaGraphConditionalHandle h, int use_handle, cudaStream_t s);
cudaError_t flow_launch_moments(int nd, int precision, bool odd, const void* f,
                                const FlowMap& fm, const Grid& g, const LbParams& lbp,
                                float* vel, double* partials, cudaStream_t s);
cudaError_t flow_launch_flags(const uint8_t* mat, long long n, int pore, uint8_t* flag,
                              cudaStream_t s);
// imap[cells[k]] = k, then cells[k] rewritten from the voxel index to the
// packed coordinates of fm (imap must hold -1 everywhere before).
cudaError_t flow_launch_imap(int* cells, int nf, int* imap, const Grid& g, int ys, int xs,
                             cudaStream_t s);
// The pull tables of fm (cells and imap ready) into nbr,
// flow_nbr_bytes(Q, fm.nf) bytes.
cudaError_t flow_launch_nbr(int nd, const FlowMap& fm, const Grid& g, int* nbr, cudaStream_t s);
cudaError_t flow_launch_final_reduce(const double* partials, int nblocks, double* out,
                                     cudaStream_t s);
int flow_blocks(long long n);
// order-preserving compaction of a 0/1 flag array (adr.cu): with idx == NULL
// only counts (cnt: one int per 1024 flags, *total on the device)
cudaError_t adr_launch_compact(const uint8_t* mflag, long long n, int* cnt, long long* total,
                               int* idx, cudaStream_t s);

// Sets what prt_last_error(NULL) returns on the calling thread (runtime.cu).
void set_noctx_error(const char* msg);

// Kernel launchers (adr.cu) -------------------------------------------------
struct AdrDev {
    Grid g;
    FastDiv div_z, div_y;  // by nz and by ny (coordinates of a voxel index)
    int nd;
    int ns;
    int has_bf;  // the run has a biofilm material code (else no biofilm flag is set)
    const uint32_t* flags;
    const float* face[3];
    float* buf[2];
    float* ladder;              // slot s at ladder + s * ns * n
    const int* slot_of_step;    // -1 or ladder slot for step n
    const int* idx;             // compressed solute voxel list
    long long nm;               // solute voxels
    PairTree tree;
    float* tree_vals;           // ns * (nleaf + ninner)
    ProgressRec* log;
    int log_cap;
};

cudaError_t adr_launch_setup(const uint8_t* mat, const float* vel, const prt_adr_params& p,
                             const AdrDev& d, cudaStream_t s);
cudaError_t adr_launch_step(const AdrDev& d, const prt_adr_params& p, AdrCtrl* ctrl,
                            int kstep, cudaStream_t s);
cudaError_t adr_launch_means(const AdrDev& d, AdrCtrl* ctrl, int slot_or_neg, float* means_out,
                             cudaStream_t s);
cudaError_t adr_launch_stop(const AdrDev& d, AdrCtrl* ctrl, const float* means,
                            cudaGraphConditionalHandle h, int use_handle, cudaStream_t s);

// Batched solves (batch.cu, batch_adr.cu, engine.cu) ------------------------
// A work-list entry: the blocks [b0, b0 + nb) of job `job` (kFlowThreads
// slots per block for flow, 256 solute voxels for transport).
struct BatchTile {
    int job;
    int b0;
    int nb;
    int pad;
};

// One flow solve of a batch: what the single-solve kernels take as
// arguments, plus the per-job convergence partials and an arrival counter
// (tile blocks finished in the current iteration; the block that completes
// the count advances the control block).
struct FlowJob {
    void* f;
    FlowMap fm;
    Grid g;
    LbParams kc;
    FlowCtrl* ctrl;
    double* partials;  // one per block of slots, as in the single solve
    unsigned* arrive;
    long long g0;      // the job has run (batch steps done) - g0 iterations
    int nb;            // blocks of slots of the job
    int pad;
};

// Solute voxels per block of a batched transport job.
constexpr int kBatchAdrBlock = 256;

// One transport solve of a batch.  Its solute voxels are cut into nbk blocks
// of kBatchAdrBlock.  On a check step each block sums the pairwise-tree
// leaves that lie inside it; a leaf that crosses the seam between blocks
// b - 1 and b is summed by whichever of the two finishes second (counter
// cnt[1 + b]), and the block that completes the job's arrival count
// (cnt[0]) forms the means, applies the stop rule and advances the control
// block.  The counters are back at zero after every step.
struct AdrJob {
    AdrDev d;
    prt_adr_params p;
    AdrCtrl* ctrl;
    float* means;          // ns floats: the pore means of the latest check
    unsigned* cnt;         // arrival counter, then one counter per seam (nbk + 1)
    const int* blk_leaf;   // nbk + 1 entries: first leaf starting in block b
    long long g0;          // the job has run (batch steps done) - g0 steps
    int nbk;
    int pad;
};

// Copy of a job descriptor into shared memory by the whole block (8-byte
// words), so per-voxel code reads its constants from shared memory.
template <class T>
__device__ __forceinline__ void block_copy(T* dst, const T* src) {
    static_assert(sizeof(T) % 8 == 0, "descriptor size must be a multiple of 8 bytes");
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(T) / 8); i += blockDim.x) d[i] = s[i];
}

// The contiguous range of work-list entries block b of g handles, so that
// consecutive tiles of a block mostly belong to one job.
__device__ __forceinline__ void tile_range(int n, int& t0, int& t1) {
    const long long b = blockIdx.x, g = gridDim.x;
    t0 = (int)(b * n / g);
    t1 = (int)((b + 1) * n / g);
}

// Each launch is persistent: `grid` blocks walk the work list, whose length
// is read on the device so a captured graph stays valid when the list is
// rewritten between replays.
// The step kernels take the batch's step counter (steps completed before
// the current graph replay) and their step's place k in the replay; a job's
// own count is that plus k minus its g0, so its control block is written
// only on the steps that sample, check or end it.
// uniform: the constants every job of the launch shares, or null.
cudaError_t batch_launch_flow(int nd, int precision, const FlowJob* jobs, const BatchTile* tiles,
                              const int* ntiles, const long long* gstep, int k,
                              const LbParams* uniform, int grid, cudaStream_t s);
int batch_flow_occupancy(int nd, int precision);
cudaError_t batch_launch_adr(int nd, int ns, const AdrJob* jobs, const BatchTile* tiles,
                             const int* ntiles, const long long* gstep, int k, int grid,
                             cudaStream_t s);
// *gstep += k: ends a graph replay of k batch steps.
cudaError_t batch_launch_gstep(long long* gstep, int k, cudaStream_t s);
int batch_adr_occupancy(int nd, int ns);
cudaError_t batch_launch_status(const int* const* done_ptrs, int n, int* out, cudaStream_t s);

}  // namespace prt
