// Host-side symbolic analysis of the batched Newton-Raphson engine.
//
// A plan is built once per (Ybus pattern, slack, PV, PQ) and holds:
//   * the Jacobian sparsity pattern, bit-exact to the reference's construction
//     (src/powerflow_algorithm/BaseNRSingleSlackAlgo.tpp:247-378 for a single slack,
//     BaseNRAlgo.tpp:396-555 for a distributed slack) and the value map from Ybus entries
//     to J entries (BaseNRSingleSlackAlgo.tpp:385-447, BaseNRAlgo.tpp:562-635);
//   * a fill-reducing column order (minimum degree on J + J^T, then the equivalent order of
//     least elimination depth, the shallowest of several relabellings) and the row pivots of a
//     threshold-partial-pivoting Gilbert-Peierls factorisation of the first Jacobian --
//     the same contract as the reference's KLU::initialize (src/linear_solvers/KLUSolver.cpp:24-45):
//     later Jacobians are refactorised with these pivots;
//   * the device schedules: the LU value layout and the phase programs of the
//     refactorisation and of both triangular solves (longest-first placement for the global-LU
//     kernels, a bank-conflict placement of the same operations for the packed shared-memory
//     layout).
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <vector>

namespace l2g {

using cplx = std::complex<double>;

// ErrorType ordinals of the reference (src/Utils.hpp:47-56).
enum Err : int {
    NoError = 0,
    SingularMatrix = 1,
    TooManyIterations = 2,
    InifiniteValue = 3,
    SolverAnalyze = 4,
    SolverFactor = 5,
    SolverReFactor = 6,
    SolverSolve = 7,
    NotInitError = 8,
    LicenseError = 9
};

struct Plan {
    // ------------------------------------------------------------ problem
    int n = 0;                        // buses
    int nnzY = 0;
    std::vector<int> Yp, Yi;          // Ybus CSC pattern
    std::vector<cplx> Yx;             // base Ybus values (CSC order)
    std::vector<int> Rp, Rj, Rrow;    // CSR copy of the pattern (row pointer, column, row)
    std::vector<int> csr_of_csc;      // CSC position -> CSR position
    std::vector<cplx> Rx;             // base values, CSR order
    bool distributed = false;
    bool dc = false;                  // DC plan: B = Re(Ybus) without the slack, no Newton loop
    int slack0 = 0;
    std::vector<int> slack_ids;
    std::vector<double> weights;      // n
    std::vector<int> mypv, pq, pvpq;  // mypv = extra slacks + pv when distributed
    int npv = 0, npq = 0, npvpq = 0, off = 0;
    int m = 0;                        // J dimension

    // ------------------------------------------------------------ Jacobian
    std::vector<int> Jp, Ji;          // J CSC pattern (bit-exact to the reference)
    std::vector<int> jsrc;            // per J entry: Ybus CSC position, -1 for a constant
    std::vector<uint8_t> jkind;       // 0 Re dS/dVa, 1 Im dS/dVa, 2 Re dS/dVm, 3 Im dS/dVm
    std::vector<double> jconst;       // value of the constant entries (distributed slack)

    // ------------------------------------------------------------ LU symbolic
    std::vector<int> q, qinv;         // column order: step k factorises J column q[k]
    std::vector<int> prow, pinv;      // row pivots: J row prow[k] is pivotal at step k
    int nnzLU = 0;
    std::vector<int> colstart;        // per step: first LU position of the column
    std::vector<int> dpos;            // per step: position of the diagonal
    std::vector<int> lstart, lcount;  // per step: L part (rows > k, ascending)
    std::vector<int> Urow_k;          // per LU position: row (step numbering)
    // Phase programs.  A program is a sequence of phases; a phase is a list of independent
    // operations (no two write the same value, none reads a value another one writes), run
    // by all threads of a CTA, with a barrier between phases.  The L columns are kept
    // undivided (L(i,c) * U(c,c)); every consumer divides by the pivot.
    // Operation (x, y, z, w | kind<<28):
    //   kind 0  lu[x] -= lu[y] * (lu[z] / lu[w])   right-looking update of column j by pivot c:
    //                                              y = undivided L(i,c), z = U(c,j), w = U(c,c)
    //   kind 2  v[x]  -= lu[y] * v[z] / lu[w]      push of an undivided column / value
    //   kind 4  v[x]  /= lu[w]                     division by a pivot
    //   kind 7  nothing (padding)
    // Operations writing the same value run on the same thread (see ProgramBuilder).
    // `factor`: refactorisation by elimination level with the forward substitution of the
    // right-hand side fused in; `backward`: U z = y; `forward`: L y = b on its own (second
    // solve of a refinement).
    struct Program {
        // 4 ints per operation (x, y, z, w | kind << 28):
        //   kind 0: LU[x] -= LU[y] * LU[z] / LU[w]   (refactorisation update, L kept undivided)
        //   kind 2: v[x]  -= LU[y] * v[z] / LU[w]    (substitution push)
        //   kind 7: empty slot
        std::vector<int> ops;
        // the same operations placed for few shared-memory bank conflicts in the packed layout
        // (same phases and widths; every written value keeps its thread and order, so the
        // results are bit-identical); empty when not built
        std::vector<int> ops_banked;
        std::vector<int> base;         // phase p = operations [base[p], base[p+1])
        std::vector<int> width;        // phase p: threads with work (the operation stride)
        int nphases() const { return (int)base.size() - 1; }
        int nops() const { return (int)(ops.size() / 4); }
    };
    Program factor, backward, forward;
    std::vector<int> colleve;         // elimination level per column
    // J fill
    std::vector<int> ytarget;         // 4 per CSR position: LU position or -1
    std::vector<int> yjpos;           // 4 per CSR position: J CSC position or -1
    std::vector<int> fillpos;         // LU positions that J does not cover
    std::vector<int> cpos;            // LU positions of constant J entries
    std::vector<double> cval;
    std::vector<int> cjpos;           // J CSC positions of constant entries
    // bus maps (positions in the permuted RHS / solution vector, -1 if absent)
    std::vector<int> xP, xQ;          // mismatch: P / Q equation of bus b -> RHS index
    std::vector<int> xVa, xVm;        // update: Va / Vm correction of bus b -> solution index
    int xSlack = -1;                  // distributed slack: solution index of slack_absorbed

    // dense tail: the last tail_k steps [tail_ct, m) form a trailing block dense enough to be
    // factorised and substituted as one dense matrix (row-major, tail_k x tail_k) instead of by
    // the phase programs, whose operations inside the block were taken out (see dense_tail)
    int tail_ct = 0, tail_k = 0;      // tail_k == 0: none
    std::vector<int> tail_map;        // tail_k^2: LU position of block entry (a, b), -1 if outside the pattern

    // statistics
    long long flops_refactor = 0;     // multiply-adds of one refactorisation
    int levels_refactor = 0, levels_fwd = 0, levels_bwd = 0;
    int bank_lanes = 0;               // lanes per bank group of the packed placement; 0: none built

    // ------------------------------------------------------------ fast decoupled
    // FDPF plan: the Ybus data above drive the mismatch; sub[0] is B' over pvpq, sub[1] B''
    // over pq (each with its own ordering, pivots, LU layout and substitution programs) and
    // sublu[k] their factor values, computed once (the matrices do not change between calls).
    // Bus maps: xP / xVa index the B' system, xQ / xVm the B'' system.
    bool fdpf = false;
    std::vector<Plan> sub;
    std::vector<std::vector<double>> sublu;
};

struct PlanOptions {
    double pivot_threshold = 1e-3;    // diagonal preference of the first factorisation
    bool fuse_forward = true;         // fuse the forward substitution into the refactorisation
    int threads = 512;                // CTA size the phase programs are laid out for
    int elem_bytes = 4;               // LU element size of the packed programs' bank placement
    bool spread_clusters = false;     // bank placement: clusters spread over a phase's slots
    int order_trials = 8;             // > 0: minimum degree of this many relabellings, each followed
                                      // by its least-depth equivalent, the shallowest kept; 0:
                                      // minimum degree only
    int level_slack = 2;              // minimum degree prefers, among the vertices of degree at most
                                      // the minimum + level_slack, the one of lowest level; 0: off
    bool dense_tail = true;           // Newton plans whose LU cannot sit in shared memory: the dense
                                      // trailing block, when there is one, becomes a dense tail
};

// Trailing blocks of at least kTailMin and at most kTailMax steps, whose LU pattern is at least
// kTailDensity full, are factorised as dense tails.
constexpr int kTailMin = 256;
constexpr int kTailMax = 768;
constexpr double kTailDensity = 0.5;

// Builds a plan.  Ybus CSC (n x n, complex), V0 and Sbus (used for the first
// factorisation's pivots).  Returns an Err code; `msg` receives a description on failure.
int build_plan(Plan &P, int n, const int *Yp, const int *Yi, const cplx *Yx, const cplx *V0, const cplx *Sbus,
               const int *slack_ids, int nslack, const double *weights, const int *pv, int npv, const int *pq,
               int npq, bool distributed, const PlanOptions &opt, std::string &msg);

// Operations packed for a shared-memory LU: the solve vector and the LU share one index
// space (v[k] -> k, a scratch slot for empty operations -> m, LU[i] -> lu_offset + i) with
// 16 bits per index, so every operation is  s[x] -= s[y] * s[z] / s[w]  (8 bytes).
int compact_lu_offset(int m);
bool compact_fits(const Plan &P);
// 2 words per op; lu_offset >= 0 places the LU elsewhere in the index space (the two systems of
// a fast-decoupled plan share one solve vector, their LUs follow it one after the other)
void compact_ops(const Plan::Program &pr, int m, std::vector<unsigned> &out, int lu_offset = -1);
// Index-space offsets of the B' and B'' LUs of a fast-decoupled plan behind their shared solve
// vector, and whether both fit the 16-bit packed indices.
void fdpf_lu_offsets(const Plan &P, int &off0, int &off1, bool &fits);
// Shared-memory wavefronts of one run of a packed program (the plan's default layout): per
// group of P.bank_lanes lanes and slot, per operand (the written word twice: loaded and stored),
// the most distinct words in one bank.  0 when the plan has no packed placement.
long long smem_wavefronts(const Plan &P, const Plan::Program &pr);

// Builds a DC plan (BaseDCAlgo, src/powerflow_algorithm/BaseDCAlgo.tpp): the matrix is
// B = Re(Ybus) over every bus except the first slack (the other slacks count as PV), factorised
// and scheduled like a Jacobian.  Ybus is the DC admittance matrix.  Returns an Err code.
int build_dc_plan(Plan &P, int n, const int *Yp, const int *Yi, const cplx *Yx, const int *slack_ids, int nslack,
                  const int *pv, int npv, const int *pq, int npq, const PlanOptions &opt, std::string &msg);

// A phase program regrouped for the instance-interleaved batch kernel, where every operation
// is run by a whole warp on 32 instances at once.  The operations of a phase are grouped by the
// value they write (a group keeps its order), groups are bin-packed onto `nwarps` warps (a warp
// runs whole groups, so no two warps write one value), and each warp's list is cut into chunks
// of `chunk` operations: chunk (round r, warp w) of phase p is chunk number phase[2p] + r *
// nwarps + w, `phase[2p+1]` rounds in all; padding operations have kind 7.
constexpr int kTileWarps = 32;  // warps of the batch-interleaved kernel (1024 threads)
constexpr int kTileChunk = 4;   // operations per warp chunk
struct TileProgram {
    std::vector<int> ops;    // 4 ints per operation, as Plan::Program
    std::vector<int> phase;  // 2 per phase: first chunk, rounds
};
void build_tile_program(const Plan::Program &pr, int nwarps, int chunk, TileProgram &out);

// A real sparse matrix, CSC (n x n, canonical).
struct RealCsc {
    const int *p, *i;
    const double *x;
};

// Builds a fast-decoupled plan (BaseFDPFAlgo, src/powerflow_algorithm/BaseFDPFAlgo.tpp:11-214):
// pvpq = [slacks after the first, pv, pq] (retrieve_pv_with_slack, BaseAlgo.hpp:201-216),
// B'_ = Bp[pvpq, pvpq] and B''_ = Bpp[pq, pq] (fill_sparse_matrices, BaseFDPFAlgo.tpp:175-214)
// from the grid-level B' and B'' (n x n), both factorised here.  Returns an Err code.
int build_fdpf_plan(Plan &P, int n, const int *Yp, const int *Yi, const cplx *Yx, const RealCsc &Bp,
                    const RealCsc &Bpp, const int *slack_ids, int nslack, const double *weights, const int *pv,
                    int npv, const int *pq, int npq, const PlanOptions &opt, std::string &msg);

// Host evaluation of the Jacobian values (J CSC order) at V for Ybus values Yx (CSC order).
void host_jacobian(const Plan &P, const cplx *Yx, const cplx *V, std::vector<double> &Jx);

}  // namespace l2g
