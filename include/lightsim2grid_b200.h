/*
 * lightsim2grid_b200.h -- C ABI of the B200 batched AC Newton-Raphson power-flow engine.
 *
 * Plain C types only: int32 indices, doubles, complex numbers as interleaved (re, im)
 * doubles, caller-owned host buffers.  No C++ exception crosses this boundary: every
 * entry point returns an int status (0 on success; otherwise the reference's ErrorType
 * ordinal, src/Utils.hpp:47-56, or -1 for invalid arguments) and pf_last_error() gives a
 * one-line description.  One plan per thread at a time; plans are not thread-safe.
 *
 * Each entry point names the reference interface it replaces (lightsim2grid 0.13.1).
 */
#ifndef LIGHTSIM2GRID_B200_H
#define LIGHTSIM2GRID_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pf_plan pf_plan;

/* Engine options.  Zero-initialised fields select the defaults. */
typedef struct pf_options {
    int precision;          /* 0: FP64 LU and solves (plain form); 1: FP32 LU and solves with
                               FP64 mismatch, update and convergence test (mixed form)        */
    int threads;            /* threads per CTA (multiple of 32; Newton plans <= 768, DC and
                               fast-decoupled plans <= 512); 0: chosen by size (Newton plans
                               of more than 4000 unknowns: 640 in the mixed form, 768 in
                               FP64)                                                        */
    int lu_placement;       /* 0 auto, 1 shared memory, 2 global memory                      */
    int fuse_forward;       /* forward substitution fused into the refactorisation program.
                               0: default (on), 1: on, 2: off                                  */
    double pivot_threshold; /* diagonal preference of the first factorisation; 0: 1e-3      */
    int fp64_fallback;      /* mixed form: re-run instances that did not converge in FP64
                               (inside the launch on the plan's own scratch, else by a second
                               launch).  0: default (on), 1: on, 2: off                         */
    int max_ctas_per_sm;    /* cap on resident CTAs per SM; 0: occupancy limit               */
    int refine;             /* mixed form: refine Newton steps once against the FP64
                               Jacobian (the one-CTA kernel skips the correction solve when
                               the FP64 residual is below tol / 100).  0: default (on), 1: on,
                               2: off                                                         */
    double refine_threshold;/* ... the steps taken from ||F||_inf below this; 0: 1e-3          */
    double lu_reuse_threshold;/* mixed form: refined steps taken from ||F||_inf below this reuse
                               the previous iteration's LU instead of refactorising (capped at
                               the refinement threshold); <= 0: never (default).  Measured at
                               1e-5: 5-9 % faster, same iterations and flags, but results up
                               to 5e-8 pu from the FP64 ones instead of 3e-10               */
    int batch_layout;       /* Newton batches of independent instances (no time-series chain):
                               0 auto: batch-interleaved for plans whose LU stays in global
                               memory with at least 60,000 entries (6,515 buses) and 4 jobs per
                               SM or more, else one CTA per instance; 1 one CTA
                               per instance; 2
                               batch-interleaved: 32 instances per CTA, one per lane, every value
                               stored as 32 consecutive per-instance values (coalesced, the batch
                               dimension amortises each phase), the last running instances of a
                               CTA and, mixed form, the FP32 failures handed to the one-CTA
                               kernel in the same stream; its per-CTA memory is allocated on
                               first use                                                     */
    int ordering;           /* elimination order of the first factorisation.  0: default, minimum
                               degree preferring low elimination levels (among the vertices of
                               degree up to the minimum + 2, the lowest level) on 8 relabellings
                               of the pattern, each followed by its equivalent reordering of least
                               depth (no added fill, fewer dependent phases), the shallowest kept;
                               1: plain minimum degree only; 2: as 0 with one labelling; 3: as 0
                               without the level preference                                    */
    int placement;          /* packed programs (LU in shared memory): 0 default = 1; 1 clusters
                               of operations writing one value spread over the phase's slots
                               (fewer bank conflicts: 2848-bus factor 36.7k -> 30.6k shared-memory
                               wavefronts, N-1 batch 11.37 -> 11.23 ms); 2 clusters in their
                               thread's first slots (shorter plan build).  Same results          */
    int level_slack;        /* orderings 0 and 2: minimum degree takes, among the vertices of
                               degree up to the minimum + level_slack, the one of lowest
                               elimination level.  0: default (2); < 0: no level preference;
                               larger values give shallower plans for some more fill          */
    int handoff_lanes;      /* batch-interleaved layout: once the jobs are exhausted, a CTA hands
                               its running instances to the one-CTA kernel when at most this many
                               of its lanes still run.  0: default (all its lanes when no lane
                               takes a second job, else half); < 0: never                      */
} pf_options;

/* DC power flow plan (BaseDCAlgo::compute_pf, src/powerflow_algorithm/BaseDCAlgo.tpp:5-175;
   the reference's DC solvers, SolverType DC / KLUDC): ybus_ri is the DC admittance matrix (CSC,
   complex); the unknowns are the angles of every bus except the first slack (further slacks
   count as PV), the matrix B = Re(Ybus) without that bus, analysed, ordered, pivoted and
   scheduled as the Newton plans are, solved in FP64.  pf_solve, pf_batch_n1, pf_batch_device and
   the scratch entry points run it: one linear solve per instance (iterations 1; max_iter and
   tol unused); the angles are shifted by the start voltage's slack angle and the magnitudes are
   the start magnitudes; a non-finite solution or one with |angle| >= 1e6 gives SolverSolve and a
   zero voltage row.  pf_get_J and pf_multi_create reject DC plans. */
int pf_dc_plan_create(int n, const int *colptr, const int *rowind, const double *ybus_ri, const int *slack_ids,
                      int nslack, const int *pv, int npv, const int *pq, int npq, const pf_options *opts,
                      pf_plan **plan);

/* Fast decoupled power flow plan (BaseFDPFAlgo::compute_pf, src/powerflow_algorithm/
   BaseFDPFAlgo.tpp:11-173; the reference's FDPF_XB_* / FDPF_BX_* solvers, src/ChooseSolver.hpp:
   21-24).  bp_* and bpp_* are the grid-level B' and B'' (n x n, real CSC) that
   GridModel::fillBp_Bpp builds for the XB or BX method (src/GridModel.cpp:1037-1064); the plan
   keeps B'[pvpq, pvpq] and B''[pq, pq] (pvpq = slacks after the first, pv, pq), factorises
   both once and uses those factors for every later call and instance, as the reference's batch
   computers do (the solver is told nothing changed after the base power flow).  Each iteration
   is a B' half-step on the angles and a B'' half-step on the magnitudes, each followed by the
   mismatch (V conj(Ybus V) - Sbus + Re(sum Sbus) w) / Vm; converged when its P (pvpq) and Q (pq)
   parts are below tol.  FP64.  pf_solve, pf_batch_n1, pf_batch_ts, pf_batch_device and the
   scratch entry points run it; pf_get_J and pf_multi_create reject it.  A singular B' or B''
   fails here with SolverFactor. */
int pf_fdpf_plan_create(int n, const int *colptr, const int *rowind, const double *ybus_ri, const int *bp_colptr,
                        const int *bp_rowind, const double *bp_x, const int *bpp_colptr, const int *bpp_rowind,
                        const double *bpp_x, const int *slack_ids, int nslack, const double *slack_weights,
                        const int *pv, int npv, const int *pq, int npq, const pf_options *opts, pf_plan **plan);

/* Sizes and schedule statistics of a plan. */
typedef struct pf_plan_info {
    int n, m, nnz_ybus, nnz_j, nnz_lu;
    int levels_refactor, levels_forward, levels_backward;
    int groups_refactor, groups_forward, groups_backward;
    long long flops_refactor;  /* multiply-adds of one refactorisation */
    int precision, threads, lu_in_shared, ctas_per_sm, grid;
    long long slab_bytes, shared_bytes;
    /* shared-memory wavefronts of one run of the factor, backward and forward programs in the
       packed layout (the LU in shared memory), from the bank model the programs are placed
       for: per group of lanes the banks serve together and per operand, the most distinct
       words in one bank.  0 when the plan's LU is not in shared memory.                       */
    long long smem_wavefronts_factor, smem_wavefronts_backward, smem_wavefronts_forward;
    /* steps of the dense tail (the trailing block factorised as one dense matrix), 0: none */
    int tail_k;
} pf_plan_info;

/* A batch whose inputs and outputs are already in device memory (pointers from
   cudaMalloc or torch).  Complex arrays are interleaved double pairs. */
typedef struct pf_device_batch {
    int n_inst;
    const void *V0;          /* complex, n per instance (or one vector if v0_stride == 0)    */
    long long v0_stride;     /* in complex elements                                          */
    const void *Sbus;        /* complex, n per instance (or one vector if sbus_stride == 0)  */
    long long sbus_stride;
    const int *ovr_ptr;      /* n_inst + 1; Ybus overrides per instance (may be NULL); at most
                                32 per instance: an instance with more is not computed
                                (errs NotInitError, iterations 0, start voltages out; a
                                time-series chain stops there)                                */
    const int *ovr_pos;      /* CSR positions of the overridden Ybus entries                  */
    const void *ovr_val;     /* complex, new value of each overridden entry                   */
    int max_iter;
    double tol;
    int chain;               /* 1: an instance starts from the previous one's solution        */
    const int *job_first;    /* njobs; instances [job_first[j], job_first[j] + job_count[j])  */
    const int *job_count;
    int njobs;
    void *Vout;              /* complex, n per instance                                       */
    int *iters;              /* n_inst                                                        */
    int *errs;               /* n_inst: ErrorType ordinals                                    */
} pf_device_batch;

/* Last error message of the calling thread. */
const char *pf_last_error(void);

/* Builds a plan: J pattern (bit-exact to the reference), fill-reducing order, pivots of the
   first factorisation at V0, device schedules; uploads the structure to the current device.
   Replaces the first-call path of BaseNRSingleSlackAlgo::compute_pf / BaseNRAlgo::compute_pf
   (src/powerflow_algorithm/BaseNRSingleSlackAlgo.tpp:76-111, BaseNRAlgo.tpp:89-116) and
   KLULinearSolver::initialize (src/linear_solvers/KLUSolver.cpp:24-45).
   Ybus: CSC (colptr n+1, rowind, values), canonical (sorted rows, no duplicates).
   distributed: 0 = single slack (KLUSolverSingleSlack), 1 = distributed slack (KLUSolver). */
int pf_plan_create(int n, const int *colptr, const int *rowind, const double *ybus_ri, const double *V0_ri,
                   const double *Sbus_ri, const int *slack_ids, int nslack, const double *slack_weights,
                   const int *pv, int npv, const int *pq, int npq, int distributed, const pf_options *opts,
                   pf_plan **out);

/* Releases a plan and its device memory. */
void pf_plan_destroy(pf_plan *plan);

/* Fills *info. */
int pf_plan_info_get(const pf_plan *plan, pf_plan_info *info);

/* Replaces the base Ybus values (same pattern).  Mirrors the reference's Ybus value
   updates between calls that keep the sparsity pattern (src/Utils.hpp:79-181, SolverControl). */
int pf_set_ybus_values(pf_plan *plan, const double *ybus_ri);

/* One power flow: BaseNRSingleSlackAlgo::compute_pf / BaseNRAlgo::compute_pf
   (src/powerflow_algorithm/BaseNRSingleSlackAlgo.tpp:12-183, BaseNRAlgo.tpp:14-186), bound as
   KLUSolverSingleSlack.solve / KLUSolver.solve (src/main.cpp:228-254).  V_out receives the
   final voltages; *converged is 1 when err == NoError. */
int pf_solve(pf_plan *plan, const double *V0_ri, const double *Sbus_ri, int max_iter, double tol, double *V_out_ri,
             int *converged, int *iters, int *err);

/* Jacobian of the last iteration of the last pf_solve, CSC.  Pass NULL arrays to get *m and
   the number of entries (returned).  Replaces get_J_python (src/main.cpp:230). */
int pf_get_J(pf_plan *plan, int *m, int *Jp, int *Ji, double *Jx);

/* Job order for an N-1 batch prepared by pf_n1_prepare (ninst solvable instances, their
   overrides ovr_ptr / ovr_pos / ovr_val_ri): instance indices by decreasing power mismatch of the
   outage at the start voltages, max over buses of |V_r conj(sum dY_rc V_c)|, a predictor of the
   iterations an instance takes.  Passing this order as the job list of a device batch starts the
   long instances first, so they do not extend the end of the launch (results do not depend on
   the order).  No counterpart in the reference (it solves the cases one after the other);
   pf_batch_n1 uses it for its own jobs. */
int pf_n1_order(const pf_plan *plan, int ninst, const int *ovr_ptr, const int *ovr_pos, const double *ovr_val_ri,
                const double *V0_ri, int *order);

/* N-1 / N-k batch: ContingencyAnalysis::compute (src/batch_algorithm/ContingencyAnalysis.cpp:166-233)
   after the base power flow.  Case c removes coef_{row,col,val}[case_ptr[c] .. case_ptr[c+1])
   from Ybus (entries must exist in the pattern).  Islanded cases (check_invertible,
   ContingencyAnalysis.cpp:14-45) are skipped: err = SingularMatrix, V row 0.  Every other case
   starts from V0.  V_out is ncases x n complex, zero for cases that did not converge.  When V_out
   is pinned host memory mapped into the device address space (cudaHostAlloc, which unified
   addressing maps), the kernel writes the rows straight into it as the cases finish; otherwise
   the rows are copied after the kernel. */
int pf_batch_n1(pf_plan *plan, int ncases, const int *case_ptr, const int *coef_row, const int *coef_col,
                const double *coef_val_ri, const double *V0_ri, const double *Sbus_ri, int max_iter, double tol,
                double *V_out_ri, int *converged, int *iters, int *errs);

/* Host preparation of an N-1 batch for pf_batch_device: islanding check and Ybus overrides
   (CSR positions, new values).  solvable[c] = 1 if case c keeps the grid connected.  Overrides
   are written for solvable cases only, compacted; returns the number of overrides written, or
   a negative status if `cap` is too small. */
int pf_n1_prepare(pf_plan *plan, int ncases, const int *case_ptr, const int *coef_row, const int *coef_col,
                  const double *coef_val_ri, int *solvable, int *ovr_ptr, int *ovr_pos, double *ovr_val_ri,
                  int cap);

/* Time series: TimeSeries::compute_Vs (src/batch_algorithm/TimeSeries.cpp:14-109).  Sbus is
   nsteps x n complex.  The steps are cut into `nchunks` contiguous chunks; inside a chunk each
   step starts from the previous step's solution, the first step of a chunk from V0 (nchunks = 1
   is the reference's exact chain).  Steps after the first divergence are not reported (V row 0,
   err = NotInitError).  Returns 0 and sets *status to 1 when every step converged. */
int pf_batch_ts(pf_plan *plan, int nsteps, const double *Sbus_ri, const double *V0_ri, int nchunks, int max_iter,
                double tol, double *V_out_ri, int *converged, int *iters, int *errs, int *status);

/* Device-resident batch on `stream` (a cudaStream_t, NULL for the default stream).  No
   host synchronisation; capturable in a CUDA graph once the plan exists (when the batch-
   interleaved layout runs -- batch_layout 2, or auto on large global-LU plans -- after one call
   of the same size outside capture: that layout's per-CTA memory is allocated on first use).
   Mixed form: a job with an instance that does not converge in FP32 is solved again in FP64
   inside the launch (option fp64_fallback), so the outputs are the FP64 outcome for those
   instances.  The current device must be the plan's (else -1, nothing launched). */
int pf_batch_device(pf_plan *plan, const pf_device_batch *batch, void *stream);

/* pf_batch_device without any allocation, for callers that cannot let the library call
   cudaMalloc (work issued during CUDA-graph stream capture, hosts that own the device-memory
   budget through their own allocator, plugin hosts that forbid allocation on work calls).
   No counterpart in the reference.  The kernel's working memory comes from a 32 MiB
   file-scope device array held on every GPU that loads the library until exit; a plan whose
   per-CTA working memory does not fit is rejected with an error, otherwise the launch uses as
   many CTAs as fit.  Mixed form: an instance that does not converge in FP32 is solved again in
   FP64 inside the launch, as pf_batch_device does (the slabs then hold an FP64 LU too, so large
   plans run on fewer CTAs: about 50 for the 2,848-bus mixed plan).  The current device must be
   the plan's (else -1, nothing launched).  The first call on a device looks the array's address
   up (cudaGetSymbolAddress) -- make it before any stream capture.  The array is shared by all
   calls and keeps the previous call's contents; the job counter is cleared before each launch.
   Calls whose kernels overlap on the GPU race on the array: keep them on one stream.  Calls no
   cudaMalloc, cudaFree or allocating library routine. */
int pf_batch_device_noalloc(pf_plan *plan, const pf_device_batch *batch, void *stream);

/* pf_batch_device with working memory supplied by the caller: `scratch` (device memory,
   256-byte aligned, `scratch_bytes` long) holds the launch's job counter and per-CTA slabs
   (pf_scratch_bytes gives the size for a number of CTAs; the launch uses as many CTAs as fit).
   Launches of one plan on different streams with disjoint scratch may overlap on the GPU: the
   plan's device data is only read.  Used by the serving loop, which admits requests against a
   device-memory budget.  Its slabs hold the FP32 solve only: instances that fail in FP32 are
   reported as they are (no FP64 fallback).  No counterpart in the reference (its solvers own
   their memory). */
int pf_batch_device_scratch(pf_plan *plan, const pf_device_batch *batch, void *scratch, long long scratch_bytes,
                            void *stream);

/* One launch over several plans (grids of different sizes), config "uneven-size batched N-1":
   batch i belongs to plans[i] (device-resident inputs and outputs, as for pf_batch_device;
   its job fields are ignored).  The launch's job list lives in device memory: job j runs
   instances [job_first[j], job_first[j] + job_count[j]) of segment job_seg[j]; CTAs take jobs
   in list order, so put the costly ones first.  The plans must share device, precision,
   refinement and LU placement; the launch uses the largest thread count, shared-memory layout
   and slab among them.  pf_multi_create uploads the segment table and allocates the scratch
   once; pf_multi_launch is asynchronous, allocates nothing and can be captured in a CUDA graph.
   No counterpart in the reference (one solver object per grid). */
typedef struct pf_multi pf_multi;
int pf_multi_create(pf_plan *const *plans, const pf_device_batch *batches, int nseg, const int *job_seg,
                    const int *job_first, const int *job_count, int njobs, pf_multi **out);
int pf_multi_launch(pf_multi *multi, void *stream);
int pf_multi_info(const pf_multi *multi, int *threads, int *grid, long long *shared_bytes,
                  long long *scratch_bytes);
void pf_multi_destroy(pf_multi *multi);

/* Branches for flow computations (BaseBatchSolverSynch::compute_amps_flows /
   compute_active_power_flows, src/batch_algorithm/BaseBatchSolverSynch.hpp:87-192): bus
   indices of both sides, the AC admittances y_ff and y_ft (complex, interleaved), the nominal
   voltage (kV) of the from bus, the in-service flag (NULL: every branch in service), sn_mva. */
typedef struct pf_branch_set {
    int nbr;
    const int *from;
    const int *to;
    const double *yff_ri;
    const double *yft_ri;
    const double *vn_kv_from;
    const unsigned char *status;
    double sn_mva;
} pf_branch_set;

/* Flows of nrows result rows on the device: amps (kA) and / or active power (MW) at the from
   side of every branch, nrows x nbr row-major (either output may be NULL).  Row r uses the
   voltages V + map[r] * v_stride (map NULL: row r; map[r] < 0, or errs[map[r]] != 0 with errs
   not NULL: all-zero voltages, giving NaN amps and 0 MW as the reference's arithmetic does).
   out_ptr / out_ids (NULL: none) list each row's removed branches, set to 0 where finite
   (ContingencyAnalysis::clean_flows, src/batch_algorithm/ContingencyAnalysis.cpp:237-250).
   Every pointer, including those in `br`, is a device pointer; bus indices must be < n.
   Asynchronous on `stream`. */
int pf_flows_device(const pf_branch_set *br, int n, int nrows, const double *V_ri, long long v_stride,
                    const int *map, const int *errs, const int *out_ptr, const int *out_ids, double *amps,
                    double *p_mw, void *stream);

/* The same from host arrays (V_ri: nrows x n complex, row-major; outputs nrows x nbr): checks
   the bus indices, copies to the device, computes, copies back and synchronises. */
int pf_flows_host(const pf_branch_set *br, int n, int nrows, const double *V_ri, const int *out_ptr,
                  const int *out_ids, double *amps, double *p_mw);

/* Ybus assembly on the device (GridModel::fillYbus, src/GridModel.cpp:676-699; branch pi-model
   src/element_container/TwoSidesContainer_rxh_A.hpp:921-940, triplets pushed per branch as ff,
   tt, ft, tf at :494-498 and summed in insertion order).  pf_ybus_positions maps (row, col)
   pairs to the plan's Ybus storage positions (-1: not in the pattern; host only).
   pf_assemble_ybus_device writes nnz values: entry p sums contributions cids[cptr[p] ..
   cptr[p+1]), each 4 * branch + kind (0 ff, 1 tt, 2 ft, 3 tf), computed from the branch's r,
   x, total shunt h (complex, split half / half) and in-service flag (NULL: all in service).
   pf_set_ybus_values_device copies such values (the plan's storage order) into the plan's
   device Ybus, asynchronously: later launches on the plan use them.  The plan's host-side
   values (pf_n1_prepare's islanding check, pf_get_J) keep what pf_plan_create or
   pf_set_ybus_values gave. */
int pf_ybus_positions(const pf_plan *plan, int ncoef, const int *rows, const int *cols, int *pos);
int pf_assemble_ybus_device(int nnz, const int *cptr, const int *cids, const double *r, const double *x,
                            const double *h_ri, const unsigned char *status, double *ybus_ri, void *stream);
int pf_set_ybus_values_device(pf_plan *plan, const double *ybus_ri, void *stream);

/* Sbus rows assembled on the device (GridModel::fillSbus_me, src/GridModel.cpp:701-716; per
   snapshot, TimeSeries::compute_Sbuses, src/batch_algorithm/TimeSeries.hpp:79-151): per bus,
   generator and static-generator active powers minus load powers (element order), divided by
   sn_mva when it differs from 1.  Bus -> element lists as CSR (n + 1 pointers each; the static
   generator lists may be NULL); injections row-major, one row per snapshot.  Device pointers;
   asynchronous. */
typedef struct pf_sbus_layout {
    int n, ngen, nsgen, nload;
    const int *gen_ptr, *gen_ids;
    const int *sgen_ptr, *sgen_ids;
    const int *load_ptr, *load_ids;
} pf_sbus_layout;
int pf_assemble_sbus_device(const pf_sbus_layout *lay, int nsteps, const double *gen_p, const double *sgen_p,
                            const double *load_p, const double *load_q, double sn_mva, double *sbus_ri,
                            void *stream);

/* Native serving core (no counterpart in the reference, which has no request loop): power-flow
   and N-1 requests over several grids, continuously batched on one GPU.  Each grid: its plan,
   base-case voltages and injections (host arrays, copied to the device once), its branch-removal
   coefficients as CSR over branches (as for pf_batch_n1) and its Newton settings.  Device memory
   is one arena of hbm_budget bytes allocated at creation; each admitted request gets one region
   of it (inputs, kernel working memory) and one of `slots` streams with pinned staging, mapped
   into the device address space: the kernel writes the results there directly.
   pf_server_submit queues a request: kind 0 = one power flow with the base injections scaled
   bus by bus by scale[n]; kind 1 = the outages of `nbranches` branches from the base-case state.
   V_out (rows x n complex, rows = 1 or nbranches), iters_out and errs_out (rows) receive the
   results in case order (islanded outages: zero row, SingularMatrix; failures: zero row).
   pf_server_poll admits queued requests oldest first while a slot is free and the arena has room,
   launches them, and writes the ids of finished requests (their outputs filled) to done_ids;
   it returns how many.  Not thread-safe: one caller thread per server. */
typedef struct pf_server pf_server;
typedef struct pf_server_grid {
    pf_plan *plan;
    const double *V0_ri;     /* base-case voltages (n complex)                     */
    const double *Sbus_ri;   /* base-case injections (n complex)                   */
    int nbr;                 /* branches                                           */
    const int *case_ptr;     /* nbr + 1: coefficients of branch b: [case_ptr[b], case_ptr[b+1]) */
    const int *rows;
    const int *cols;
    const double *vals_ri;
    int max_iter;            /* 0: 10     */
    double tol;              /* 0: 1e-8   */
} pf_server_grid;
int pf_server_create(const pf_server_grid *grids, int ngrids, long long hbm_budget, int slots, int max_instances,
                     pf_server **server);
int pf_server_submit(pf_server *server, long long id, int grid, int kind, const double *scale, int nbranches,
                     const int *branches, double *V_out, int *iters_out, int *errs_out);
int pf_server_poll(pf_server *server, long long *done_ids, int cap);
/* SM reservation of a server (no counterpart in the reference).  A request is small when its
   instances x buses are at most 20,000 on a grid of at most 2,000 buses (an instance of a larger
   grid holds its SM for a millisecond or more); a large request is admitted only while the SMs taken by
   the CTAs of the large requests in flight stay within (SMs - reserved_sms), so the reserved SMs
   stay free for small requests (stream priorities alone cannot move a resident CTA); its launch
   uses at most large_request_ctas CTAs (0: no cap), each solving several of its instances in
   turn.  Defaults: an eighth of the SMs reserved, no cap.  Takes effect for later admissions. */
int pf_server_configure(pf_server *server, int reserved_sms, int large_request_ctas);
/* Device-resident request loop (no counterpart in the reference).  enable = 1: instead of one
   launch per request, the small requests (see pf_server_configure) of each class of grids of at
   most 2,000 buses (plans with the LU in shared memory; the others) are served by a persistent
   launch of the Newton kernel that takes jobs from a ring in device memory (the large requests keep
   their own launches, which spread over the SMs the loops leave free):
   an admitted request's inputs, segment (plan and batch) and jobs are copied to the device on a
   feeder stream, then the ring's tail; the loop's CTAs claim the jobs as they appear, write the
   results into the slot's mapped pinned staging and count the finished instances per slot in
   mapped host memory, which pf_server_poll reads.  A CTA leaves after a few milliseconds without
   work (every wait in the kernel is bounded); the loop is launched again when work is published
   while it is not running.  ctas_shared / ctas_global: CTAs of each class's loop (0: a quarter of
   the SMs' worth, an eighth each when both classes exist).  Switch modes only while no request is
   queued or running.  Results are those of the launch-per-request mode, bit for bit. */
int pf_server_device_loop(pf_server *server, int enable, int ctas_shared, int ctas_global);
int pf_server_state(const pf_server *server, int *pending, int *inflight, long long *bytes_in_use);
/* Latency split of a server's finished requests of one grid and kind (no counterpart in the
   reference): out[0..1] = p50 / p99 of the admission wait (pf_server_submit to the launch or
   publication by pf_server_poll), out[2..3] = p50 / p99 of the device time (that to the
   pf_server_poll that saw the request finished), in ms of the host's steady clock; out[4] = how
   many requests (the first 262,144 per grid and kind since the last reset).  reset != 0 clears
   the figures after reading them. */
int pf_server_latency_split(pf_server *server, int grid, int kind, double *out, int reset);
void pf_server_destroy(pf_server *server);

/* Scratch bytes pf_batch_device_scratch needs to run `ctas` CTAs at once (at most the plan's
   grid); < 0 on error. */
long long pf_scratch_bytes(const pf_plan *plan, int ctas);

/* pf_batch_device, synchronously, with per-phase SM-cycle counters: out[0..7] = cycles summed
   over CTAs spent in mismatch, J fill, refactorisation, forward substitution, backward
   substitution, refinement (mixed form), voltage update / start-up, and the number of
   instances.  The device counterpart of the reference's per-phase NR timers
   (get_timers_jacobian, src/powerflow_algorithm/BaseNRAlgo.hpp:48-62).  With the batch-interleaved
   layout the counters are that kernel's (its follow-up launches are not counted), the
   substitution slots cover its backward programs and out[7] counts its rounds. */
int pf_batch_device_phase_cycles(pf_plan *plan, const pf_device_batch *batch, void *stream, double *out);

/* pf_batch_device, synchronously, recording the SM clock after every phase of the first
   Newton iteration of CTA 0's first instance: out[i] = cycles since the first mark (the
   marks follow the J fill, then every phase of the refactorisation, backward and, when the
   step is refined, forward and backward programs, then the update).  Returns the number of
   marks (<= cap).  A diagnostic of the phase programs' critical path. */
int pf_batch_device_phase_trace(pf_plan *plan, const pf_device_batch *batch, void *stream, double *out, int cap);

/* Timers of the last call (seconds): [0] total, [1] host preparation, [2] host->device,
   [3] kernel, [4] device->host, [5] instances re-solved in FP64 by the mixed form's fallback,
   inside the launch or by a second launch (count, as a double).
   Replaces get_timers (src/main.cpp:236) and the batch timers (src/main.cpp:1174-1178). */
int pf_timers(const pf_plan *plan, double *out, int nout);

/* ---- host diagnostics (no device needed) ---------------------------------------------- */

/* Jacobian sparsity pattern the engine builds for this problem (CSC), as the reference's
   fill_jacobian_matrix_unkown_sparsity_pattern (BaseNRSingleSlackAlgo.tpp:247-378,
   BaseNRAlgo.tpp:396-555).  Pass NULL Jp / Ji to get *m and the entry count (returned). */
int pf_host_jacobian_pattern(int n, const int *colptr, const int *rowind, const double *ybus_ri,
                             const int *slack_ids, int nslack, const double *slack_weights, const int *pv,
                             int npv, const int *pq, int npq, int distributed, int *m, int *Jp, int *Ji);

/* Runs the device schedules (refactorisation update lists and level order, forward and
   backward substitution level order) sequentially on the host: factorises J(V) with the pivots
   chosen at V0 and solves J x = b.  b and x are in J row / column numbering (length m).  Also
   checks that the packed, bank-placed (for 4- and 8-byte words) and batch-interleaved forms of
   the programs give the results of the plain ones.  Used to test a plan's schedules on machines
   without a GPU. */
int pf_host_schedule_solve(int n, const int *colptr, const int *rowind, const double *ybus_ri, const double *V0_ri,
                           const double *V_ri, const int *slack_ids, int nslack, const double *slack_weights,
                           const int *pv, int npv, const int *pq, int npq, int distributed, const double *b,
                           double *x, pf_plan_info *info);

#ifdef __cplusplus
}
#endif

#endif /* LIGHTSIM2GRID_B200_H */
