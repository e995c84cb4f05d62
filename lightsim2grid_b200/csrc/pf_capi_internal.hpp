// Internal interfaces between the translation units behind the C ABI (not part of the ABI).
#pragma once

#include <cstddef>
#include <string>

#include "../../include/lightsim2grid_b200.h"
#include "pf_engine.cuh"

namespace l2g {

// Kernel arguments of a device-resident batch (scratch, counter and variant not yet set).
BatchArgs device_args(const pf_device_batch *b);

// pf_batch_device with caller-provided scratch: the first 256 bytes hold the job counter,
// the rest the per-CTA slabs (the grid shrinks to the slabs that fit).  Allocates nothing.
// fp64_fallback: a mixed plan that runs its FP64 fallback inside launches does so here too, with
// slabs of plan_fallback_slab_bytes (else the FP32 result of a failing instance is reported as is).
// Fails without launching when the current device is not the plan's.
int batch_device_with_scratch(pf_plan *pl, const pf_device_batch *b, void *stream, void *scratch,
                              size_t scratch_bytes, bool fp64_fallback);

// Bytes of one CTA slab of the plan's kernel.
size_t plan_slab_bytes(const pf_plan *pl);

// Bytes of one CTA slab when the launch runs the FP64 fallback inside (plan_slab_bytes when the plan
// has no such fallback).
size_t plan_fallback_slab_bytes(const pf_plan *pl);

// Device the plan was created on (-1 for a null plan).
int plan_device(const pf_plan *pl);

// Device-resident request loop over several plans (the serving core's device loop): the shape of
// one persistent launch of the Newton kernel in queue mode.  The plans must share device,
// precision, refinement and LU placement; the shape takes the largest thread count, shared memory
// and slab, with room for the in-launch FP64 fallback when every plan has it.
struct LoopShape {
    int device = 0, precision = 0, threads = 0, num_sms = 0, ctas_per_sm = 0;
    bool lu_in_smem = false, refine = false, inline_fb = false;
    size_t smem = 0, slab = 0;
};
int loop_shape(pf_plan *const *plans, int n, LoopShape *sh);
// The segment of one request (its plan and device batch) for a loop whose per-CTA slabs start at
// `scratch`.
int loop_segment(pf_plan *pl, const pf_device_batch *b, const LoopShape &sh, unsigned char *scratch, Segment *seg);
// One persistent launch of `grid` CTAs taking jobs from q (asynchronous on `stream`).
int loop_launch(const LoopShape &sh, const Segment &seg0, const DevQueue &q, int grid, void *stream);

// Sets the message returned by pf_last_error on this thread.
void set_last_error(const std::string &msg);

}  // namespace l2g
