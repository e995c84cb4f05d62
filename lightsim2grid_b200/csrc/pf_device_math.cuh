// Device arithmetic shared by the batch kernels: complex helpers, the Jacobian entries of one
// Ybus entry, and the quotient used by the LU programs.
#pragma once

#include <cuda_runtime.h>

namespace l2g {
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double cabs2(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

constexpr double kPi = 3.141592653589793;

// dS/dVa and dS/dVm of Ybus entry (r, c), as BaseNRAlgo::_dSbus_dV (BaseNRAlgo.tpp:228-257)
__device__ __forceinline__ void dsbus(double2 y, double2 vr, double2 vc, bool diag, double2 ib, double &dvar,
                                      double &dvai, double2 &dvm) {
    const double ic = 1.0 / cabs2(vc);
    const double2 vnc = make_double2(vc.x * ic, vc.y * ic);
    double2 a = cmul(cconj(cmul(y, vnc)), vr);  // conj(Y * Vnorm_c) * V_r
    double2 b = cmul(y, vc);                    // Y * V_c
    if (diag) {
        const double ir = 1.0 / cabs2(vr);
        const double2 vnr = make_double2(vr.x * ir, vr.y * ir);
        const double2 t = cmul(cconj(ib), vnr);
        a.x += t.x;
        a.y += t.y;
        b.x -= ib.x;
        b.y -= ib.y;
    }
    dvar = b.x * vr.y - b.y * vr.x;  // conj(-b) * (j V_r)
    dvai = -(b.x * vr.x + b.y * vr.y);
    dvm = a;
}

// a / b: correctly rounded in FP64; in FP32 (mixed form) the reciprocal-based quotient
// (within 2 ulp), whose error the FP64-residual refinement of the Newton step absorbs
__device__ __forceinline__ double lu_div(double a, double b) { return a / b; }
__device__ __forceinline__ float lu_div(float a, float b) { return __fdividef(a, b); }

}  // namespace
}  // namespace l2g
