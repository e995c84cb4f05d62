// Ybus and Sbus assembled on the GPU from element data.
//
// Ybus (GridModel::fillYbus, src/GridModel.cpp:676-699, with the branch pi-model of
// src/element_container/TwoSidesContainer_rxh_A.hpp:921-940 and the half / half shunt split of
// LineContainer.cpp:27-33): per branch k in service, ys = 1 / (r + j x), y_ff = ys + h/2,
// y_tt = ys + h/2, y_ft = y_tf = -ys; the four coefficients of every branch are summed into the
// Ybus entries (f,f), (t,t), (f,t), (t,f).  The host lists, for every stored Ybus entry, its
// contributions (4 * branch + kind) in the order the reference's triplets sum them; the kernel
// gathers them in that order (no atomics: the same bits on every run).
//
// Sbus (GridModel::fillSbus_me, src/GridModel.cpp:701-716; per snapshot as
// TimeSeries::compute_Sbuses, src/batch_algorithm/TimeSeries.hpp:79-151): per bus, generator
// and static-generator active powers minus load powers, in element order, divided by sn_mva
// when it differs from 1.
#include "pf_assembly.cuh"

#include <algorithm>
#include <cmath>

namespace l2g {
namespace {

__device__ __forceinline__ double2 branch_coef(const YbusArgs &A, int c) {
    const int k = c >> 2, kind = c & 3;
    if (A.status && !A.status[k]) return make_double2(0.0, 0.0);
    const double r = A.r[k], x = A.x[k];
    const double den = r * r + x * x;
    const double2 ys = make_double2(r / den, -x / den);  // 1 / (r + j x)
    if (kind >= 2) return make_double2(-ys.x, -ys.y);     // ft, tf
    const double2 h = A.h[k];                             // ff, tt: ys + h / 2
    return make_double2(ys.x + 0.5 * h.x, ys.y + 0.5 * h.y);
}

__global__ void assemble_ybus_kernel(const YbusArgs A) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < A.nnz; p += gridDim.x * blockDim.x) {
        double2 y = make_double2(0.0, 0.0);
        const int c1 = A.cptr[p + 1];
        for (int c = A.cptr[p]; c < c1; ++c) {
            const double2 v = branch_coef(A, A.cids[c]);
            y.x += v.x;
            y.y += v.y;
        }
        A.out[p] = y;
    }
}

__global__ void assemble_sbus_kernel(const SbusArgs A) {
    const long long total = (long long)A.nsteps * A.n;
    const bool scale = fabs(A.sn_mva - 1.0) > 1e-7;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / A.n), b = (int)(i - (long long)s * A.n);
        double2 v = make_double2(0.0, 0.0);
        for (int e = A.gen_ptr[b]; e < A.gen_ptr[b + 1]; ++e) v.x += A.gen_p[(long long)s * A.ngen + A.gen_ids[e]];
        for (int e = A.sgen_ptr ? A.sgen_ptr[b] : 0; A.sgen_ptr && e < A.sgen_ptr[b + 1]; ++e)
            v.x += A.sgen_p[(long long)s * A.nsgen + A.sgen_ids[e]];
        for (int e = A.load_ptr[b]; e < A.load_ptr[b + 1]; ++e) {
            const long long q = (long long)s * A.nload + A.load_ids[e];
            v.x -= A.load_p[q];
            v.y -= A.load_q[q];
        }
        if (scale) {
            v.x /= A.sn_mva;
            v.y /= A.sn_mva;
        }
        A.out[i] = v;
    }
}

}  // namespace

cudaError_t launch_assemble_ybus(const YbusArgs &A, int num_sms, cudaStream_t st) {
    if (A.nnz <= 0) return cudaSuccess;
    assemble_ybus_kernel<<<std::min((A.nnz + 255) / 256, num_sms * 8), 256, 0, st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_assemble_sbus(const SbusArgs &A, int num_sms, cudaStream_t st) {
    const long long total = (long long)A.nsteps * A.n;
    if (total <= 0) return cudaSuccess;
    const long long blocks = std::min<long long>((total + 255) / 256, (long long)num_sms * 16);
    assemble_sbus_kernel<<<(int)blocks, 256, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace l2g
