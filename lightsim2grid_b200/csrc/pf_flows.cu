// Branch flows of a batch of power-flow results on the GPU.
//
// Restates BaseBatchSolverSynch::compute_amps_flows / compute_active_power_flows
// (src/batch_algorithm/BaseBatchSolverSynch.hpp:87-192) for AC results and
// ContingencyAnalysis::clean_flows (src/batch_algorithm/ContingencyAnalysis.cpp:237-250):
//   I_ft = conj(y_ff E_f + y_ft E_t),  S_ft = E_f I_ft
//   amps = |S_ft| sn_mva / (sqrt(3) |E_f| vn_kv(from))   [kA]
//   p    = Re(S_ft) sn_mva                                [MW]
// A branch out of service keeps 0 (the reference skips it in zeroed matrices); a result row
// whose voltages are all zero (a failed or islanded case) gives NaN amps (0 / 0) and 0 MW, as
// the reference's arithmetic does; clean_flows then sets each case's removed branches to 0
// where the value is finite.
//
// Layout: one CTA per result row; the row's outputs are written coalesced, its voltages are
// gathered per branch end, the per-branch data comes from L2.
#include "pf_flows.cuh"

#include <algorithm>
#include <cmath>

namespace l2g {
namespace {

__device__ __forceinline__ double2 cmulf(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Source row of result row r (-1: zero voltages).
__device__ __forceinline__ int source_row(const FlowArgs &A, int r) {
    int src = A.map ? A.map[r] : r;
    if (src >= 0 && A.errs && A.errs[src] != 0) src = -1;  // failed instance: zero voltages
    return src;
}

// Flows of one branch at one row's voltages ef (from) and et (to).
__device__ __forceinline__ void branch_flow(double2 yf, double2 yt, double vn, double sn, double2 ef, double2 et,
                                            double &a, double &p) {
    const double sqrt3 = 1.7320508075688772;
    const double2 i1 = cmulf(yf, ef), i2 = cmulf(yt, et);
    const double2 ift = make_double2(i1.x + i2.x, -(i1.y + i2.y));  // conj
    const double2 s = cmulf(ef, ift);
    const double vf_kv = sqrt(ef.x * ef.x + ef.y * ef.y) * vn;
    a = sqrt(s.x * s.x + s.y * s.y) * sn / (sqrt3 * vf_kv);
    p = s.x * sn;
}

// One CTA per row (grid-stride over rows); each thread takes every blockDim-th branch and
// gathers its two voltages through L1 (a row's voltages stay cached while the CTA works on it).
// Measured on the 2848-bus N-1 flows (3776 x 3776): 0.18 ms; staging the row, or tiles of rows,
// in shared memory was slower (0.19 / 0.27 ms: fewer CTAs per SM in flight).
__global__ void __launch_bounds__(256) branch_flows_kernel(const FlowArgs A) {
    for (int row = blockIdx.x; row < A.nrows; row += gridDim.x) {
        const int src = source_row(A, row);
        const double2 *V = src >= 0 ? A.V + (long long)src * A.v_stride : nullptr;
        const int o0 = A.out_ptr ? A.out_ptr[row] : 0, o1 = A.out_ptr ? A.out_ptr[row + 1] : 0;
        for (int k = threadIdx.x; k < A.nbr; k += blockDim.x) {
            double a = 0.0, p = 0.0;
            if (A.status == nullptr || A.status[k]) {
                const int f = A.from[k], t = A.to[k];
                const double2 ef = V ? V[f] : make_double2(0.0, 0.0);
                const double2 et = V ? V[t] : make_double2(0.0, 0.0);
                branch_flow(A.yff[k], A.yft[k], A.vn_kv_from[k], A.sn_mva, ef, et, a, p);
            }
            // clean_flows: the branches removed in this row's case are 0 where finite
            for (int o = o0; o < o1; ++o)
                if (A.out_ids[o] == k) {
                    if (isfinite(a)) a = 0.0;
                    if (isfinite(p)) p = 0.0;
                }
            if (A.amps) A.amps[(long long)row * A.nbr + k] = a;
            if (A.p_mw) A.p_mw[(long long)row * A.nbr + k] = p;
        }
    }
}

}  // namespace

cudaError_t launch_branch_flows(const FlowArgs &A, int num_sms, cudaStream_t st) {
    if (A.nrows <= 0 || A.nbr <= 0) return cudaSuccess;
    branch_flows_kernel<<<std::min(A.nrows, num_sms * 8), 256, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace l2g
