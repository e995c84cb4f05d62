// Device-side data of the batched Newton-Raphson engine (shared by the kernels and the
// host orchestration).  Plain pointers only: the structure arrays are uploaded once per
// plan; the batch arrays are per call.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace l2g {

// Structure arrays of one plan on the device (see pf_plan.hpp for their meaning).
struct DevPlan {
    int n, m, nnzY, nnzLU, distributed;
    const int *Rp, *Rj, *Rrow;
    const double2 *Rx;
    const double *w;
    const int4 *ytarget;   // 4 LU positions per CSR position
    const int4 *yjpos;     // 4 J positions per CSR position
    const int *fillpos;
    int nfill;
    const int *cpos, *cjpos;
    const double *cval;
    int nconst;
    const int *xP, *xQ, *xVa, *xVm;
    int xSlack;
    const double *wJ;        // distributed slack: J(P(r), 0) per bus (0 if none)
    // phase programs (see pf_plan.hpp): operations as int4 (x, y, z, w | kind << 28) and
    // phase boundaries; factor includes the forward substitution of the right-hand side
    const int4 *fac_ops, *bwd_ops, *fwd_ops;
    const int *fac_base, *bwd_base, *fwd_base;
    const int *fac_width, *bwd_width, *fwd_width;
    int fac_nph, bwd_nph, fwd_nph;
    // packed operations of the shared-memory layout (x and LU in one index space)
    int compact, lu_offset;
    const uint2 *fac_cops, *bwd_cops, *fwd_cops;
    // narrow phases of the packed programs (shared-memory LU): phases [nar_a[k], nar_b[k]) of
    // program k (0 factor, 1 backward, 2 forward) run on the first nar_warps warps only, between
    // barriers of those warps, with their operations staged in shared memory once per plan
    int nar_a[3], nar_b[3], nar_warps;
    int nar_first[3];   // program k's operation index of the first staged operation (base[nar_a])
    int nar_off[4];     // staged operations of program k at [nar_off[k], nar_off[k + 1])
    const int *dpos;         // pivot position per column (m)
    int dc, slack0;          // DC plan (B = Re(Ybus) without the slack) and its slack bus
    const double *luval;     // constant factor values (LU layout) of a fast-decoupled system
    // the phase programs regrouped for the batch-interleaved kernel (TileProgram, pf_plan.hpp):
    // operations (kind 7 padding) and, per phase, the first chunk and the number of rounds
    const int4 *tfac_ops, *tbwd_ops, *tfwd_ops;
    const int *tfac_phase, *tbwd_phase, *tfwd_phase;
    // dense tail (global-memory LU plans): steps [tail_ct, tail_ct + tail_k) factorised and
    // substituted as one dense row-major block in the CTA's slab; tail_map: LU position of each
    // block entry (-1 outside the pattern)
    int tail_ct, tail_k;
    const int *tail_map;
};

// One batch launch.
struct BatchArgs {
    int n_inst;
    const double2 *V0;        // start voltages; instance i reads V0 + i * v0_stride
    long long v0_stride;      // 0: one start point shared by all instances
    const double2 *Sbus;      // injections; instance i reads Sbus + i * sbus_stride
    long long sbus_stride;
    const int *ovr_ptr;       // per-instance Ybus overrides (CSR positions / new values), may be null
    const int *ovr_pos;
    const double2 *ovr_val;
    int max_iter;
    double tol;
    const int *job_first;     // jobs: instances [job_first[j], job_first[j] + job_count[j])
    const int *job_count;
    int njobs;
    int chain;                // 1: an instance starts from the previous instance's solution
    int *job_counter;         // zero before the launch
    double2 *Vout;            // n per instance
    int *iters;
    int *errs;
    double *Jout;             // J values (CSC order) of the last iteration of instance j_inst
    int j_inst;
    unsigned char *scratch;   // per-CTA slab
    long long slab_bytes;
    int lu_in_smem;
    int refine;               // FP32 LU only: one FP64-residual refinement of every Newton step
    double refine_below;      // ... taken when ||F||_inf before the step is below this
    double reuse_below;       // refined steps from ||F||_inf below this reuse the previous LU (0: never)
    unsigned long long *phase_cycles;  // optional, kPhaseSlots per CTA: SM cycles per phase
    unsigned long long *trace;         // optional: CTA 0, first Newton iteration of its first
                                       // instance: clock after every phase of every program
    int trace_cap;
    int tile_lanes;                    // batch-interleaved kernel: lanes (instances) per CTA
    // hand-off from the batch-interleaved kernel to the one-CTA kernel (no host synchronisation):
    int *hand_list, *hand_count;       // instances continued from their current state (stragglers)
    int hand_lanes;                    // ... once the jobs are exhausted and at most this many of a
                                       // CTA's lanes are still running
    int *fb_list, *fb_count;           // mixed form: instances that failed in FP32, re-solved in FP64
    const int *njobs_dev;              // one-CTA kernel: job count in device memory (min with njobs)
    const int *it_start;               // ... iterations an instance has already taken (null: 0)
    int v0_from_out;                   // ... an instance starts from its output row (its state)
    const int *vout_row;               // optional: output row of each instance (default: the instance)
    int zero_failed;                   // 1: an instance that did not converge writes a zero row
    int fp64_inline;                   // mixed form: a job that failed in FP32 is solved again in FP64
                                       // by the same CTA (slab_bytes then holds an FP64 LU, and the
                                       // dynamic shared memory an FP64 solve vector)
};

// The output row of an instance (Vout may be mapped host memory: rows stream out as instances
// finish).
__device__ __forceinline__ double2 *out_row(const BatchArgs &A, int inst, int n) {
    return A.Vout + (long long)(A.vout_row ? A.vout_row[inst] : inst) * n;
}

// One segment of a launch over several plans: a plan and its batch (device memory).
struct alignas(16) Segment {
    DevPlan P;
    BatchArgs A;
};

// Launch over several plans (segments): job j runs instances [job_first[j], job_first[j] +
// job_count[j]) of segment job_seg[j].  segs == nullptr: a launch of one plan.
// Device-resident request loop: a persistent launch takes its jobs from a ring in device memory
// that the host appends to (through copies on a stream of its own), one segment per request slot.
struct QueueJob {
    int slot;   // the request's segment (and completion counter)
    int first;  // its instances [first, first + count)
    int count;
    int req;    // the request's sequence number: identifies the segment a CTA holds
};
struct DevQueue {
    const QueueJob *jobs;   // ring of `cap` jobs
    int cap;
    const Segment *segs;    // one per slot
    int *head;              // jobs claimed (device memory, advanced with atomicCAS)
    const int *tail;        // jobs published (device memory, written by the host's copies)
    int *done;              // per slot, instances finished (mapped host memory, system-scope adds)
    int *closing;           // device memory: set, the CTAs leave once the ring is empty
    int idle_polls;         // a CTA that polled an empty ring this many times sets `closing` and
                            // leaves (bounded wait): the launch ends as a whole, so the host never
                            // sees a launch that kept only some of its CTAs
};

struct MultiArgs {
    const Segment *segs;
    const int *job_seg;
    const int *job_first;
    const int *job_count;
    int njobs;
    int *job_counter;
    DevQueue q;             // q.jobs non-null: the request loop (segs, job lists unused)
};

// phase_cycles slots: mismatch, J fill, refactorisation, forward, backward, refinement,
// update, instances
constexpr int kPhaseSlots = 8;

constexpr int kMaxOverrides = 32;

// Bytes of the per-CTA global slab and of the dynamic shared memory.
size_t slab_bytes(const DevPlan &P, int lu_bytes, bool lu_in_smem);
size_t smem_bytes(const DevPlan &P, int lu_bytes, int x_bytes, bool lu_in_smem);

// precision: 0 = FP64 LU and solves, 1 = FP32 LU and solves (FP64 mismatch and update).
// A.lu_in_smem and A.refine select the kernel variant.
cudaError_t launch_nr_batch(const DevPlan &P, const BatchArgs &A, int precision, int threads, int grid,
                            size_t smem, cudaStream_t stream, const MultiArgs &M = MultiArgs{});
// Copies the converged result rows of a compacted batch into case order (zero rows for
// cases with map[c] < 0 or errs[map[c]] != 0).
cudaError_t launch_scatter_case_rows(const double2 *src, const int *errs, const int *map, int ncases, int n,
                                     double2 *dst, int num_sms, cudaStream_t st);
// Resident CTAs per SM for a configuration (0 if it cannot launch).
int nr_occupancy(int precision, bool lu_in_smem, bool refine, int threads, size_t smem);

// Raises a kernel's dynamic shared-memory limit to the device's maximum (once per kernel and device).
cudaError_t allow_max_smem(const void *fn);

// Batch-interleaved Newton-Raphson (pf_tile.cu): 32 instances per CTA, one per lane, every value
// stored as 32 consecutive per-instance values; one CTA of 512 threads per SM.  precision as
// launch_nr_batch; A.scratch holds `grid` slabs of tile_slab_bytes; chain must be 0.
cudaError_t launch_nr_tile(const DevPlan &P, const BatchArgs &A, int precision, int grid, cudaStream_t stream);
size_t tile_slab_bytes(const DevPlan &P, int lu_bytes);
size_t tile_smem_bytes(const DevPlan &P);

// Fast decoupled power flow of a batch: P carries the Ybus rows, slack weights and bus maps,
// B0 / B1 the substitution programs and constant factors of B' and B''.  lu_in_smem: both
// factors are copied into every CTA's shared memory (else read from global memory).
// ctas_per_sm: the residency the launch was configured for (selects the register budget of
// the 128-thread variants: up to 4 per SM unconstrained, more with 64 registers).
cudaError_t launch_fdpf_batch(const DevPlan &P, const DevPlan &B0, const DevPlan &B1, const BatchArgs &A,
                              int threads, int ctas_per_sm, int grid, size_t smem, cudaStream_t stream);
size_t fdpf_smem_bytes(const DevPlan &B0, const DevPlan &B1, bool lu_in_smem);
size_t fdpf_slab_bytes(const DevPlan &P);
// resident CTAs per SM of the variant chosen for (lu_in_smem, threads, wanted ctas_per_sm; 0: most)
int fdpf_occupancy(bool lu_in_smem, int threads, int ctas_per_sm, size_t smem);

}  // namespace l2g
