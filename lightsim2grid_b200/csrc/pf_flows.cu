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
// Layout: one CTA per result row (grid-stride over rows).  The row's voltages are read once,
// coalesced, into shared memory (when they fit), the per-branch data comes from L2, and the
// outputs of the row are written coalesced: the kernel streams each row's voltages in and its
// flows out.
#include "pf_flows.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <set>

namespace l2g {
namespace {

__device__ __forceinline__ double2 cmulf(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <bool V_SMEM>
__global__ void __launch_bounds__(256) branch_flows_kernel(const FlowArgs A) {
    extern __shared__ __align__(16) double2 vrow[];
    const double sqrt3 = 1.7320508075688772;
    for (int row = blockIdx.x; row < A.nrows; row += gridDim.x) {
        int src = A.map ? A.map[row] : row;
        if (src >= 0 && A.errs && A.errs[src] != 0) src = -1;  // failed instance: zero voltages
        const double2 *V = src >= 0 ? A.V + (long long)src * A.v_stride : nullptr;
        if (V_SMEM) {
            __syncthreads();  // the previous row's readers are done
            for (int b = threadIdx.x; b < A.n; b += blockDim.x) vrow[b] = V ? V[b] : make_double2(0.0, 0.0);
            __syncthreads();
        }
        const int o0 = A.out_ptr ? A.out_ptr[row] : 0, o1 = A.out_ptr ? A.out_ptr[row + 1] : 0;
        double *amps = A.amps ? A.amps + (long long)row * A.nbr : nullptr;
        double *pmw = A.p_mw ? A.p_mw + (long long)row * A.nbr : nullptr;
        for (int k = threadIdx.x; k < A.nbr; k += blockDim.x) {
            double a = 0.0, p = 0.0;
            if (A.status == nullptr || A.status[k]) {
                const int f = A.from[k], t = A.to[k];
                double2 ef, et;
                if (V_SMEM) {
                    ef = vrow[f];
                    et = vrow[t];
                } else {
                    ef = V ? V[f] : make_double2(0.0, 0.0);
                    et = V ? V[t] : make_double2(0.0, 0.0);
                }
                const double2 yf = A.yff[k], yt = A.yft[k];
                const double2 i1 = cmulf(yf, ef), i2 = cmulf(yt, et);
                const double2 ift = make_double2(i1.x + i2.x, -(i1.y + i2.y));  // conj
                const double2 s = cmulf(ef, ift);
                const double vf_kv = sqrt(ef.x * ef.x + ef.y * ef.y) * A.vn_kv_from[k];
                a = sqrt(s.x * s.x + s.y * s.y) * A.sn_mva / (sqrt3 * vf_kv);
                p = s.x * A.sn_mva;
            }
            // clean_flows: the branches removed in this row's case are 0 where finite
            for (int o = o0; o < o1; ++o)
                if (A.out_ids[o] == k) {
                    if (isfinite(a)) a = 0.0;
                    if (isfinite(p)) p = 0.0;
                }
            if (amps) amps[k] = a;
            if (pmw) pmw[k] = p;
        }
    }
}

}  // namespace

size_t flows_smem_bytes(int n) {
    const size_t b = (size_t)n * sizeof(double2);
    return b <= kFlowsSmemMax ? b : 0;
}

cudaError_t launch_branch_flows(const FlowArgs &A, int num_sms, cudaStream_t st) {
    if (A.nrows <= 0 || A.nbr <= 0) return cudaSuccess;
    const size_t smem = flows_smem_bytes(A.n);
    const int grid = std::min(A.nrows, num_sms * 8);
    if (smem > 0) {
        // the shared-memory limit of the staged variant is raised once per device
        static std::mutex mu;
        static std::set<int> done;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        {
            std::lock_guard<std::mutex> lk(mu);
            if (!done.count(dev)) {
                e = cudaFuncSetAttribute(branch_flows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFlowsSmemMax);
                if (e != cudaSuccess) return e;
                done.insert(dev);
            }
        }
        branch_flows_kernel<true><<<grid, 256, smem, st>>>(A);
    } else {
        branch_flows_kernel<false><<<grid, 256, 0, st>>>(A);
    }
    return cudaGetLastError();
}

}  // namespace l2g
