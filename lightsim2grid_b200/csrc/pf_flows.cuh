// Branch flows of a batch of power-flow results (see pf_flows.cu).
#pragma once

#include <cuda_runtime.h>

namespace l2g {

// One launch: rows of results (a case or a snapshot each), branches, outputs.  All pointers
// are device pointers.
struct FlowArgs {
    const double2 *V;        // voltages; row r reads V + src(r) * v_stride (n values)
    long long v_stride;      // in complex values
    const int *map;          // row -> source row (-1: no result, zero voltages); null: identity
    const int *errs;         // per source row: nonzero = failed, zero voltages (may be null)
    int nrows, n;
    const int *from, *to;    // per branch: bus indices
    const double2 *yff, *yft;
    const double *vn_kv_from;
    const unsigned char *status;  // per branch: in service (null: all)
    int nbr;
    double sn_mva;
    const int *out_ptr;      // nrows + 1: branches removed in each row's case (may be null)
    const int *out_ids;
    double *amps;            // nrows x nbr, row-major (may be null)
    double *p_mw;            // nrows x nbr, row-major (may be null)
};

cudaError_t launch_branch_flows(const FlowArgs &A, int num_sms, cudaStream_t st);

}  // namespace l2g
