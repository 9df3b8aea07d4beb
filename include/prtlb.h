/*
 * prtlb.h -- C ABI of the B200 PRT-LB solver (libprtlb.so).
 *
 * The reference (PRT-LB, a pure NumPy simulator) has no native interface; its
 * callers import three Python functions by name:
 *
 *   stokes_d2q9   3D/tools/prtlb_2d.py:348   D2Q9 TRT Stokes flow
 *   stokes_d3q19  3D/tools/prtlb_3d.py:348   D3Q19 TRT Stokes flow
 *   solve_adr     3D/tools/prtlb_3d.py:781   finite-volume ADR + reactions
 *                 (byte-identical copy at 3D/tools/prtlb_2d.py:812)
 *
 * Every entry point below is what a ctypes binding of those functions binds.
 * The Python package prtlb_gpu wraps them with the reference's signatures.
 *
 * Conventions
 *   - Plain C types only.  Host pointers are borrowed for the duration of the
 *     call; device memory is owned by the context.
 *   - Every call returns PRT_OK (0) or a negative status; prt_last_error()
 *     gives the message.  No C++ exception crosses this boundary.
 *   - One context = one CUDA device + one stream.  Calls on one context are
 *     serialised by the caller; different contexts may run concurrently.
 *   - Grids are C-ordered material arrays: (nx, ny) in 2D, (nx, ny, nz) in 3D,
 *     material code 2 = pore (the reference's PORE, prtlb_3d.py SOLID/WALL/PORE).
 */
#ifndef PRTLB_H
#define PRTLB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PRT_ABI_VERSION 1
#define PRT_MAX_SPECIES 8

/* status codes */
#define PRT_OK 0
#define PRT_E_INVALID (-1)   /* bad argument (the reference raises ValueError) */
#define PRT_E_CUDA (-2)      /* a CUDA call failed */
#define PRT_E_OOM (-3)       /* device allocation failed */
#define PRT_E_STATE (-4)     /* call made out of order (e.g. run before begin) */
#define PRT_E_CANCELLED (-5) /* the progress callback asked to stop */
#define PRT_E_NODEV (-6)     /* no CUDA device */

/* population storage for the flow solve */
#define PRT_FP64 0     /* float64, as the reference                             */
#define PRT_FP32 1     /* float32 holding f_i - w_i; momentum and antisymmetric
                          non-equilibrium part in float64, the rest in float32  */
#define PRT_FP16 2     /* float16 holding (f_i - w_i) * 2^k, collided in float32 */
#define PRT_FP32_F32 3 /* float32 holding f_i - w_i, collided in float32        */

typedef struct prt_ctx prt_ctx;

/* ABI version of the loaded library (PRT_ABI_VERSION at build time). */
int prt_abi_version(void);

/* Create a context on CUDA device `device`.  *out is NULL on failure. */
int prt_create(int device, prt_ctx** out);

/* Release every device buffer of the context and the context itself. */
void prt_destroy(prt_ctx* ctx);

/* Message of the last failed call on ctx (ctx == NULL: the last failed call
 * without a context on this thread, prt_create or prt_flow_noalloc). */
const char* prt_last_error(const prt_ctx* ctx);

/* Number of kernels this context has launched so far (graph nodes included). */
int64_t prt_kernel_launches(const prt_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order or time
 * their own work around the solver's. */
void* prt_stream(const prt_ctx* ctx);

/* Device time of the last solve's time loops, from CUDA events recorded on
 * the context's stream around them: out[0] flow loop ms, out[1] its
 * iterations, out[2] transport loop ms, out[3] its steps. */
int prt_last_timing(const prt_ctx* ctx, double* out4);

/* sizeof of the ABI structs, for binding checks (needs no GPU):
 * 0 prt_flow_params, 1 prt_flow_info, 2 prt_adr_params,
 * 3 prt_adr_run_params, 4 prt_adr_result, 5 prt_adr_geom,
 * 6 prt_adr_stats, 7 prt_physics_stats; anything else: 0. */
size_t prt_sizeof(int which);

/* ------------------------------------------------------------------------ */
/* Flow: stokes_d2q9 / stokes_d3q19                                         */
/* ------------------------------------------------------------------------ */

/* Arguments of stokes_d3q19(g, nit, force, tau_lb, magic, tol, info)
 * (prtlb_3d.py:348) and stokes_d2q9 (prtlb_2d.py:348). */
typedef struct prt_flow_params {
    int32_t nd;        /* 2 (D2Q9) or 3 (D3Q19) */
    int32_t dims[3];   /* nx, ny, nz (nz ignored when nd == 2) */
    int64_t nit;       /* iteration CAP, FlowConvergence max_it */
    double force;      /* body force along +x, lattice units */
    double tau;        /* relaxation time, > 0.5 */
    double magic;      /* TRT magic parameter Lambda (3/16) */
    double tol;        /* stop when the relative change of mean|u_x| per
                          `every` iterations is <= tol; tol <= 0: never */
    int32_t every;     /* convergence check interval (50), must be even */
    int32_t precision; /* PRT_FP64 / PRT_FP32 / PRT_FP16 */
} prt_flow_params;

/* What the solve reports (FlowConvergence.report, prtlb_3d.py:237, plus the
 * FP64 reductions the reference does not have). */
typedef struct prt_flow_info {
    int64_t iters;         /* flow_iters */
    int32_t converged;     /* flow_converged */
    int32_t pad0;
    double change;         /* flow_change (inf when never evaluated) */
    int64_t fluid_cells;   /* pore voxels */
    int64_t nonfinite;     /* non-finite float32 velocity components */
    double umax;           /* max float32 speed over pore voxels */
    double speed_sum;      /* FP64 sum of float32 speed over pore voxels */
    double ux_sum;         /* FP64 sum of u_x over pore voxels (pre-cast) */
    double mass;           /* FP64 sum of rho over pore voxels */
    double permeability;   /* nu * <u_x>_V / force, voxel^2, <>_V over ALL cells */
    double fp16_scale;     /* 2^k scale used by PRT_FP16 (1 otherwise) */
} prt_flow_info;

/* Host buffers: mat (nx*ny[*nz] uint8), vel_out (3*nx*ny[*nz] float32,
 * component-major, zero in solid; in 2D vel_out[2] == 0). */
int prt_flow(prt_ctx* ctx, const uint8_t* mat, const prt_flow_params* p,
             float* vel_out, prt_flow_info* info);

/* Same, with DEVICE pointers (already resident on the context's device). */
int prt_flow_dev(prt_ctx* ctx, const uint8_t* d_mat, const prt_flow_params* p,
                 float* d_vel_out, prt_flow_info* info);

/* The flow solve for callers that cannot allocate device memory.  No
 * counterpart in the reference: it exists for hosts that own the device
 * memory pool (a framework that forbids foreign cudaMalloc, a real-time loop
 * that must not block on the allocator, a plug-in host that hands out
 * buffers but no allocator).  The caller passes d_mat and d_vel_out as
 * device pointers it owns and a cudaStream_t (NULL: the default stream); no
 * context is needed and nothing is allocated or freed.  All other scratch
 * (both lattices, masks, partial sums, control block) is one 48 MiB
 * file-scope __device__ array in the library, which every GPU that loads
 * the library holds until exit; a grid that does not fit (64^3 D3Q19 at
 * float32 does) is refused with PRT_E_INVALID and a message giving both
 * sizes.  Every call looks up the array's address on the current device
 * (cudaGetSymbolAddress) and runs there; nothing is cached between calls.
 * Calls share the array: calls that overlap on the GPU race and must be
 * serialised.  The call returns after its work on the stream has finished,
 * also when it fails after its first launch.  Errors are read with
 * prt_last_error(NULL), which a successful call leaves empty. */
int prt_flow_noalloc(const uint8_t* d_mat, const prt_flow_params* p, float* d_vel_out,
                     prt_flow_info* info, void* stream);

/* ------------------------------------------------------------------------ */
/* Transport: solve_adr (prtlb_3d.py:781-1595)                              */
/* ------------------------------------------------------------------------ */

/* Everything the time loop needs, already reduced to float32 lattice numbers
 * by the host exactly as solve_adr's set-up computes them (9.1-9.3). */
typedef struct prt_adr_params {
    int32_t nd;
    int32_t dims[3];
    int32_t ns;                 /* chemicals */
    uint32_t moving_mask;       /* bit j: chemical j is transported */
    uint32_t pinned_mask;       /* bit j: moving and fed (inlet not NaN) */
    int32_t pore_code;          /* 2 */
    int32_t biofilm_code;       /* material code of biofilm voxels, -1: none */
    float u_scale;              /* float32 velocity scale (mean axial or speed) */
    float dt;                   /* float32 time step */
    float feed[PRT_MAX_SPECIES];
    /* initial condition: 0 zero, 1 every solute voxel, 2 biofilm voxels only */
    int32_t init_mode[PRT_MAX_SPECIES];
    float init_value[PRT_MAX_SPECIES];
    /* harmonic face diffusivities, float32: [pore|pore, pore|biofilm, biofilm|biofilm] */
    float dface[PRT_MAX_SPECIES][3];
    /* biotic dual-Monod (rate_biotic, prtlb_3d.py:1224) */
    int32_t biotic_on;
    float k;                    /* Da / l_ref */
    int32_t ks_donor_pos;       /* ks_donor > 0 */
    float ks_donor;
    int32_t ks_acceptor_pos;    /* ks_acceptor > 0 */
    float ks_acceptor;
    int32_t coupled;            /* biomass_coupled and ns > 3 and c_init[3] > 0 */
    float c3_init;
    float neg_alpha;            /* float32(-alpha) */
    int32_t alpha_cap;          /* ns > 1 and alpha > 0 */
    float alpha_dt;             /* float32(float32(alpha) * dt) */
    float prod_coef;            /* float32(1 - (yield if ns > 3 else 0)) */
    float yield_;               /* float32(yield) */
    float kd;                   /* biomass decay, lattice */
    /* abiotic first order (rate_abiotic, prtlb_3d.py:1271) */
    int32_t abio_on;            /* ka > 0 and abiotic_index < ns */
    int32_t j_ab;               /* abiotic_index */
    int32_t j_mk;               /* abiotic_product_index, -1: none */
    float ka;
    int32_t surface_only;
    /* reversible sorption (new term, no reference counterpart):
       r = k_sorp * (C[j_c] - C[j_s] / K_d), dC[j_c] -= r, dC[j_s] += r */
    int32_t sorp_on;
    int32_t j_c;
    int32_t j_s;
    float k_sorp;
    float inv_kd_sorp;
    int32_t pad1;
} prt_adr_params;

/* Progress callback: solve_adr's on_progress(step, limit, mean, change).
 * Return non-zero to cancel the run (PRT_E_CANCELLED). */
typedef int (*prt_progress_cb)(void* user, int64_t step, int64_t limit,
                               double mean0, double change);

typedef struct prt_adr_run_params {
    int64_t limit;        /* steps if given, else max_steps */
    int32_t until_conv;   /* 1: steps is None (stop rule active) */
    int32_t check;        /* max(int(1/dt), 100) */
    double tol;           /* solve_adr tol */
    double ratio;         /* snapshot ladder ratio (1.12) */
} prt_adr_run_params;

typedef struct prt_adr_result {
    int64_t steps;        /* n at exit */
    int32_t hit_cap;      /* until_conv and n >= limit */
    int32_t ladder;       /* snapshots kept (len(keep_steps)) */
    int64_t checks;       /* convergence checks evaluated */
    double last_rest;     /* rest of the last check (inf if none) */
} prt_adr_result;

/* Which voxels hold solute: pore, plus biofilm when a biofilm code is set
 * (solve_adr 9.1, prtlb_3d.py:831-846). */
typedef struct prt_adr_geom {
    int32_t nd;
    int32_t dims[3];
    int32_t pore_code;    /* 2 */
    int32_t biofilm_code; /* -1: none */
} prt_adr_geom;

/* What solve_adr's set-up reads from the velocity field, over the solute
 * voxels m, in float32 with numpy's summation order (prtlb_3d.py:860-865,
 * 977-978): vel[0][m].mean(), sqrt(sum_a vel[a]^2)[m].mean(), max |vel[a]|. */
typedef struct prt_adr_stats {
    int64_t solute_voxels;
    int64_t biofilm_voxels;
    float mean_axial;
    float mean_speed;
    float vmax[3];
    float pad;
} prt_adr_stats;

/* Stage 1 of a transport solve: take the material grid and the flow field
 * (float32, (3, grid) component-major as stokes_* returns), build the voxel
 * flags and the summation tree, and return the velocity statistics the host
 * needs to derive the time step.  Host buffers are copied; device buffers
 * are borrowed until prt_adr_begin returns. */
int prt_adr_stage(prt_ctx* ctx, const uint8_t* mat, const float* vel,
                  const prt_adr_geom* geom, prt_adr_stats* stats);
int prt_adr_stage_dev(prt_ctx* ctx, const uint8_t* d_mat, const float* d_vel,
                      const prt_adr_geom* geom, prt_adr_stats* stats);

/* Stage 2: with the lattice numbers, build the face velocities, the initial
 * state and ladder snapshot 0.  The geometry must match the staged one. */
int prt_adr_begin(prt_ctx* ctx, const prt_adr_params* p);

/* Run the time loop.  cb may be NULL. */
int prt_adr_run(prt_ctx* ctx, const prt_adr_run_params* rp, prt_progress_cb cb,
                void* user, prt_adr_result* res);

/* Ladder step numbers (keep_steps), count written to *count. */
int prt_adr_ladder(prt_ctx* ctx, int64_t* steps, int32_t cap, int32_t* count);

/* Copy ladder snapshot `slot` ((ns, grid) float32) to host / device memory. */
int prt_adr_fetch(prt_ctx* ctx, int32_t slot, float* out);
int prt_adr_fetch_dev(prt_ctx* ctx, int32_t slot, float* d_out);

/* Per-species float32 pore means of snapshot `slot`, computed with numpy's
 * float32 pairwise summation order (what solve_adr's check uses). */
int prt_adr_means(prt_ctx* ctx, int32_t slot, float* means);

/* Ends the transport state of the context.  Device buffers of up to
 * 256 MiB each stay with the context for its next transport run (so
 * back-to-back solves skip the allocator); larger ones are freed. */
int prt_adr_end(prt_ctx* ctx);

/* Frees every transport buffer of the context (prt_destroy does too). */
int prt_adr_release(prt_ctx* ctx);

/* ------------------------------------------------------------------------
 * Batched and served solves.  No counterpart in the reference, which runs
 * one solve at a time (build_dataset_3d.py loops over rocks and calls
 * stokes_d3q19 then solve_adr for each).  A solve is split into set-up
 * (prt_flow_start / prt_adr_start), a time loop that a batch runs together
 * with other solves, and results (prt_flow_finish / prt_adr_finish).  The
 * loop of a batched solve is bit-identical to prt_flow / prt_adr_run on the
 * same inputs, whatever else is in the batch.
 * ------------------------------------------------------------------------ */

/* Sets up the flow solve of prt_flow on ctx without running its loop; the
 * material grid is copied from the host. */
int prt_flow_start(prt_ctx* ctx, const uint8_t* mat, const prt_flow_params* p);

/* Final field and info of a started flow solve whose loop has finished.
 * vel_out is a host buffer as in prt_flow, or NULL to keep the field on the
 * device only (for prt_adr_stage_flow). */
int prt_flow_finish(prt_ctx* ctx, float* vel_out, prt_flow_info* info);

/* prt_adr_stage_dev on the material grid and final field of the context's
 * own flow solve (after prt_flow_finish). */
int prt_adr_stage_flow(prt_ctx* ctx, const prt_adr_geom* geom, prt_adr_stats* stats);

/* Frees the flow lattices and maps of ctx (keeps the material grid and the
 * field staged for transport).  A context in a batch may call it once its
 * flow solve is finished (prt_flow_finish). */
int prt_flow_release(prt_ctx* ctx);

/* Sets up the transport run of prt_adr_run (after prt_adr_begin) without
 * running its loop; no progress callback. */
int prt_adr_start(prt_ctx* ctx, const prt_adr_run_params* rp);

/* Result of a started transport run whose loop has finished; afterwards
 * prt_adr_ladder / prt_adr_fetch work as after prt_adr_run. */
int prt_adr_finish(prt_ctx* ctx, prt_adr_result* res);

/* Concurrent solves: enqueue the whole flow loop of a started solve
 * (prt_flow_start), or the whole transport loop of a started run
 * (prt_adr_start), on the context's own stream and return at once; many
 * contexts then run side by side on one GPU, each loop as one CUDA graph.
 * prt_ctx_busy reports whether the enqueued loop is still running; the
 * results are read with prt_flow_finish / prt_adr_finish (which wait). */
int prt_flow_launch(prt_ctx* ctx);
int prt_adr_launch(prt_ctx* ctx);
int prt_ctx_busy(prt_ctx* ctx, int32_t* busy);

typedef struct prt_batch prt_batch;

/* A batch on CUDA device `device`, with its own stream.  Each step advances
 * every running job by one flow iteration or one transport step, all jobs
 * in one persistent launch per (lattice, precision) or (dimension, species)
 * class, over a work list of tiles (128-voxel blocks for flow, 256 for
 * transport); steps run as a CUDA graph of
 * `graph_steps` steps (0: 20). */
int prt_batch_create(int device, int32_t graph_steps, prt_batch** out);

/* Waits for the batch's work and frees it; the jobs are left as they are. */
void prt_batch_destroy(prt_batch* b);

const char* prt_batch_last_error(const prt_batch* b);

/* Adds a context whose flow solve was started (prt_flow_start) or whose
 * transport run was started (prt_adr_start); it joins at the next launch.
 * A context is in one batch at a time, on the batch's device, and must not
 * be used by other calls until it is collected or removed. */
int prt_batch_add(prt_batch* b, prt_ctx* job);

/* Takes a job out of the batch (not needed for collected jobs), between
 * launches.  A batch keeps its jobs' iteration / step counts implicitly and
 * writes them to a job's control block only on the steps that check or end
 * it, so removing an unfinished job writes its count back; it can then join
 * another batch (prt_batch_add) and go on from where it was. */
int prt_batch_remove(prt_batch* b, prt_ctx* job);

/* Enqueues `steps` batch steps and returns without waiting. */
int prt_batch_launch(prt_batch* b, int32_t steps);

/* Waits for the enqueued steps; *n_done = jobs whose loop has finished. */
int prt_batch_wait(prt_batch* b, int32_t* n_done);

/* prt_batch_launch then prt_batch_wait. */
int prt_batch_run(prt_batch* b, int32_t steps, int32_t* n_done);

/* Moves up to `cap` finished jobs out of the batch into out[] (after a
 * wait); *count = how many. */
int prt_batch_collect(prt_batch* b, prt_ctx** out, int32_t cap, int32_t* count);

/* Jobs in the batch (pending additions included). */
int prt_batch_size(const prt_batch* b, int32_t* flow_jobs, int32_t* adr_jobs);

/* Tile size in blocks (1, 2 or 4) and grid: a persistent grid of
 * grid_mult (1 or 2) resident waves walking the work list, or 0 for one
 * block per work-list entry; tile_blocks 0 = choose both by timing the
 * first launches. */
int prt_batch_tune(prt_batch* b, int32_t tile_blocks, int32_t grid_mult);

/* out8: kernel launches, graph builds, tile blocks, grid multiple, steps
 * run, last launch ms (device), tiles of the last launch, 0. */
int prt_batch_stats(const prt_batch* b, double* out8);

/* Free and total memory of CUDA device `device` (cudaMemGetInfo), for
 * admission control; errors via prt_last_error(NULL). */
int prt_mem_info(int device, uint64_t* free_bytes, uint64_t* total_bytes);

/* ------------------------------------------------------------------------
 * Geometry preparation, once per rock before its solves.
 * ------------------------------------------------------------------------ */

/* The walk from the inlet face through the pore space: for every voxel of
 * the grid `mat` (nd 2 or 3, dims as in prt_flow_params, C order), the
 * fewest face-neighbour steps (6 in 3D, 4 in 2D, not periodic) from a voxel
 * of material pore_code on the face where axis inlet_axis is 0 to it, through
 * voxels of that material.  steps_out (host, one int32 per voxel) gets the
 * count for every reached pore voxel, -1 for voxels of another material and
 * -2 for pore the walk never reaches; *n_reached / *n_pore (either may be
 * NULL) the reached and all pore voxels.  One walk replaces three reference
 * routines: keep_inlet_connected (prtlb_3d.py:530-563; its scipy components
 * touching the face are the reached set), geodesic_steps
 * (prt_core/conventions.py:72-115) and the relaxed geodesic of the practice
 * dataset (build_practice_dataset.py:53-73, whose converged value it is). */
int prt_inlet_walk(prt_ctx* ctx, const uint8_t* mat, int32_t nd, const int32_t* dims,
                   int32_t pore_code, int32_t inlet_axis, int32_t* steps_out,
                   int64_t* n_reached, int64_t* n_pore);

/* The same walk seeded on the plane where axis `axis` equals `plane`
 * (0 <= plane < dims[axis]) instead of the face; it runs both ways along the
 * axis.  A pore component touches planes p and q exactly when the walk from
 * p reaches plane q: the percolation checks of the dataset builders,
 * percolates_3d (build_dataset_3d.py:281-286), percolates
 * (build_dataset_2d.py:290-294), _percolates and keep_percolating_cluster
 * (build_geometry_3d.py:201-221). */
int prt_walk_from_plane(prt_ctx* ctx, const uint8_t* mat, int32_t nd, const int32_t* dims,
                        int32_t pore_code, int32_t axis, int32_t plane, int32_t* steps_out,
                        int64_t* n_reached, int64_t* n_pore);

/* Material codes of a solid grid (label_materials, build_geometry_3d.py:
 * 224-239): `solid` (host, one byte per voxel, nonzero = solid, nd 2 or 3,
 * dims as in prt_flow_params) gives mat_out (host, uint8 per voxel) = 2 for
 * pore, 1 for solid with a pore face neighbour (the bounce-back wall), 0 for
 * the other solid.  Positions beyond the grid's faces count as solid. */
int prt_label_materials(prt_ctx* ctx, const uint8_t* solid, int32_t nd, const int32_t* dims,
                        uint8_t* mat_out);

/* ------------------------------------------------------------------------
 * check_physics (prtlb_3d.py:1632-1843) on the device: the statistics its
 * rules read, reduced from snapshots out (n_t, ns, voxels) float32 on the
 * device, with the material grid (pore where mat == pore_code).  The rules
 * and messages are the host's (prtlb_gpu.physics.check_physics(...,
 * on_gpu=True)); results that stay on the device are judged without a copy.
 * ------------------------------------------------------------------------ */
#define PRT_PHYS_MAX_SNAPSHOTS 256

typedef struct prt_physics_stats {
    int64_t n_nan, n_inf;        /* over the whole result */
    int64_t n_triples, n_flips;  /* last donor snapshot: pore triples along x and
                                    those whose neighbour differences change sign */
    int32_t has_pore[PRT_MAX_SPECIES];   /* any non-NaN pore value seen */
    float pore_max[PRT_MAX_SPECIES];     /* over the pore of every snapshot */
    float pore_min[PRT_MAX_SPECIES];
    float final_absmax[PRT_MAX_SPECIES]; /* max |value| over the pore of the last one */
    float mid_max[PRT_PHYS_MAX_SNAPSHOTS];  /* donor, plane x = nx / 2, per snapshot */
    float end_max[PRT_PHYS_MAX_SNAPSHOTS];  /* donor, plane x = nx - 1 */
} prt_physics_stats;

/* Copies a host result out (n_t, ns, voxels) and its material grid into the
 * context; the three calls below then take d_out = NULL / d_mat = NULL for
 * them (until the next stage or inlet walk on the context). */
int prt_physics_stage(prt_ctx* ctx, const float* out, const uint8_t* mat, int32_t nd,
                      const int32_t* dims, int32_t n_t, int32_t ns);

int prt_physics_stats_dev(prt_ctx* ctx, const float* d_out, const uint8_t* d_mat, int32_t nd,
                          const int32_t* dims, int32_t n_t, int32_t ns, int32_t pore_code,
                          prt_physics_stats* stats);

/* Donor against chemical j (1 <= j < ns) over the pore of every snapshot:
 * moments6 = {count, mean0, mean_j, var0, var_j, cov} (population, float64). */
int prt_physics_moments_dev(prt_ctx* ctx, const float* d_out, const uint8_t* d_mat, int32_t nd,
                            const int32_t* dims, int32_t n_t, int32_t ns, int32_t pore_code,
                            int32_t j, double* moments6);

/* max |a_j - scale a_0| over the same voxels, in float32 as numpy forms it. */
int prt_physics_maxdev_dev(prt_ctx* ctx, const float* d_out, const uint8_t* d_mat, int32_t nd,
                           const int32_t* dims, int32_t n_t, int32_t ns, int32_t pore_code,
                           int32_t j, float scale, float* maxdev);

/* Host helper, no GPU: the placement loop of the seeded ball packs used as
 * synthetic rocks (prtlb_gpu.geometry.random_pack).  No counterpart in the
 * reference (its build_spheres, build_geometry_3d.py:129-150, makes
 * overlapping spheres).  solid: uint8 grid of `shape` (nd 2 or 3) to stamp;
 * cand: ncand rows of nd+1 uniform numbers (centre / L, radius fraction);
 * centres (cap x nd) / radii (cap) hold the placed balls; state = {balls,
 * consecutive rejections, tries, solid voxels}, read and updated.  Places
 * until the solid fraction reaches target_frac, the tries reach max_tries,
 * the candidates run out or `cap` balls are placed.  Returns the candidates
 * consumed, or a negative status. */
int64_t prt_pack_balls(uint8_t* solid, int32_t nd, const int32_t* shape, const double* cand,
                       int64_t ncand, double rmin, double rmax, double target_frac,
                       int64_t overlap_after, int64_t max_tries, double* centres,
                       double* radii, int64_t cap, int64_t* state);

#ifdef __cplusplus
}
#endif

#endif /* PRTLB_H */
