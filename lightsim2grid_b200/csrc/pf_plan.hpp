// Host-side symbolic analysis of the batched Newton-Raphson engine.
//
// A plan is built once per (Ybus pattern, slack, PV, PQ) and holds:
//   * the Jacobian sparsity pattern, bit-exact to the reference's construction
//     (src/powerflow_algorithm/BaseNRSingleSlackAlgo.tpp:247-378 for a single slack,
//     BaseNRAlgo.tpp:396-555 for a distributed slack) and the value map from Ybus entries
//     to J entries (BaseNRSingleSlackAlgo.tpp:385-447, BaseNRAlgo.tpp:562-635);
//   * a fill-reducing column order (minimum degree on J + J^T) and the row pivots of a
//     threshold-partial-pivoting Gilbert-Peierls factorisation of the first Jacobian --
//     the same contract as the reference's KLU::initialize (src/linear_solvers/KLUSolver.cpp:24-45):
//     later Jacobians are refactorised with these pivots;
//   * the device schedules: the LU value layout, the per-column update lists of the
//     left-looking refactorisation and the level sets of the refactorisation and of both
//     triangular solves.
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

// One group of elimination levels.  kind 0: a "wide" level, its items are spread over
// all warps and a block barrier follows.  kind 1: a chain of levels with few items each,
// run by warp 0 alone, in order, with warp barriers only.
struct LevelGroup {
    int begin;   // first item (index into the item order array)
    int end;     // one past the last item
    int kind;    // 0 wide, 1 chain
    int lanes;   // lanes cooperating on one item (solves only): 1, 2, 4, 8, 16 or 32
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
    // Right-looking refactorisation.  An update group (c, j) applies pivot c to column j:
    // A(i, j) -= A(i, c) * U(c, j) / U(c, c) for every row i of L(:, c).  Groups of one
    // elimination level are independent except when they write the same entry; they are
    // coloured into conflict-free phases.  The divisions L(:, c) /= U(c, c) of a level run
    // at the start of the next level's first phase (they touch no entry that phase uses).
    std::vector<int> grp_lstart, grp_lcount, grp_upos, grp_dpos, grp_dst;  // per group
    std::vector<int> dst;             // destination positions, grp_dst[g] .. + grp_lcount[g]
    struct Phase {
        int gbeg, gend;               // update groups
        int dbeg, dend;               // division entries
        int lanes;                    // lanes per group (1..32)
    };
    std::vector<Phase> phases;
    std::vector<int> div_pos, div_dpos;  // L entry and its pivot, per division entry
    std::vector<int> colleve;         // elimination level per column
    // triangular solves (row oriented)
    std::vector<int> lrow_ptr, lrow_col, lrow_pos;   // L(i, k < i)
    std::vector<int> urow_ptr, urow_col, urow_pos;   // U(i, k > i)
    std::vector<int> fwd_order, bwd_order;
    std::vector<LevelGroup> fwd_groups, bwd_groups;
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

    // statistics
    long long flops_refactor = 0;     // multiply-adds of one refactorisation
    int levels_refactor = 0, levels_fwd = 0, levels_bwd = 0;
};

struct PlanOptions {
    double pivot_threshold = 1e-3;    // diagonal preference of the first factorisation
    int chain_max_items = 2;          // solve levels with at most this many rows join a chain
    int warps = 16;                   // warps per CTA the schedules are sized for
};

// Builds a plan.  Ybus CSC (n x n, complex), V0 and Sbus (used for the first
// factorisation's pivots).  Returns an Err code; `msg` receives a description on failure.
int build_plan(Plan &P, int n, const int *Yp, const int *Yi, const cplx *Yx, const cplx *V0, const cplx *Sbus,
               const int *slack_ids, int nslack, const double *weights, const int *pv, int npv, const int *pq,
               int npq, bool distributed, const PlanOptions &opt, std::string &msg);

// Host evaluation of the Jacobian values (J CSC order) at V for Ybus values Yx (CSC order).
void host_jacobian(const Plan &P, const cplx *Yx, const cplx *V, std::vector<double> &Jx);

}  // namespace l2g
