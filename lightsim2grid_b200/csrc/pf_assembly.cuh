// Ybus and Sbus assembled on the GPU from element data (see pf_assembly.cu).
#pragma once

#include <cuda_runtime.h>

namespace l2g {

// Ybus values of a fixed pattern: entry p sums contributions cids[cptr[p] .. cptr[p+1]) in that
// order; contribution c = 4 * branch + kind (0 ff, 1 tt, 2 ft, 3 tf).  Device pointers.
struct YbusArgs {
    int nnz;
    const int *cptr, *cids;
    const double *r, *x;
    const double2 *h;               // total branch shunt, split half / half
    const unsigned char *status;    // null: all in service
    double2 *out;                   // nnz values
};

// Sbus rows (nsteps x n): per bus, generators and static generators minus loads, in element
// order (bus -> element lists as CSR), injections row-major per step.  Device pointers.
struct SbusArgs {
    int nsteps, n;
    int ngen, nsgen, nload;
    const int *gen_ptr, *gen_ids, *sgen_ptr, *sgen_ids, *load_ptr, *load_ids;
    const double *gen_p, *sgen_p, *load_p, *load_q;
    double sn_mva;
    double2 *out;
};

cudaError_t launch_assemble_ybus(const YbusArgs &A, int num_sms, cudaStream_t st);
cudaError_t launch_assemble_sbus(const SbusArgs &A, int num_sms, cudaStream_t st);

}  // namespace l2g
