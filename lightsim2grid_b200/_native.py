"""ctypes binding of the C ABI declared in include/lightsim2grid_b200.h.

The library is built in-tree by ``lightsim2grid_b200.build``.  There is no fallback:
when the library is missing or no CUDA device is present the calls raise.
"""
import ctypes
import os

import numpy as np

from .build import LIB

_lib = None

i32p = ctypes.POINTER(ctypes.c_int32)
f64p = ctypes.POINTER(ctypes.c_double)


class PfOptions(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("threads", ctypes.c_int), ("lu_placement", ctypes.c_int),
                ("fuse_forward", ctypes.c_int), ("pivot_threshold", ctypes.c_double),
                ("fp64_fallback", ctypes.c_int), ("max_ctas_per_sm", ctypes.c_int), ("refine", ctypes.c_int),
                ("refine_threshold", ctypes.c_double), ("lu_reuse_threshold", ctypes.c_double),
                ("batch_layout", ctypes.c_int), ("ordering", ctypes.c_int), ("placement", ctypes.c_int),
                ("level_slack", ctypes.c_int), ("handoff_lanes", ctypes.c_int)]


class PfPlanInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("m", ctypes.c_int), ("nnz_ybus", ctypes.c_int), ("nnz_j", ctypes.c_int),
                ("nnz_lu", ctypes.c_int), ("levels_refactor", ctypes.c_int), ("levels_forward", ctypes.c_int),
                ("levels_backward", ctypes.c_int), ("groups_refactor", ctypes.c_int),
                ("groups_forward", ctypes.c_int), ("groups_backward", ctypes.c_int),
                ("flops_refactor", ctypes.c_longlong), ("precision", ctypes.c_int), ("threads", ctypes.c_int),
                ("lu_in_shared", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("grid", ctypes.c_int),
                ("slab_bytes", ctypes.c_longlong), ("shared_bytes", ctypes.c_longlong),
                ("smem_wavefronts_factor", ctypes.c_longlong), ("smem_wavefronts_backward", ctypes.c_longlong),
                ("smem_wavefronts_forward", ctypes.c_longlong), ("tail_k", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PfDeviceBatch(ctypes.Structure):
    _fields_ = [("n_inst", ctypes.c_int), ("V0", ctypes.c_void_p), ("v0_stride", ctypes.c_longlong),
                ("Sbus", ctypes.c_void_p), ("sbus_stride", ctypes.c_longlong), ("ovr_ptr", ctypes.c_void_p),
                ("ovr_pos", ctypes.c_void_p), ("ovr_val", ctypes.c_void_p), ("max_iter", ctypes.c_int),
                ("tol", ctypes.c_double), ("chain", ctypes.c_int), ("job_first", ctypes.c_void_p),
                ("job_count", ctypes.c_void_p), ("njobs", ctypes.c_int), ("Vout", ctypes.c_void_p),
                ("iters", ctypes.c_void_p), ("errs", ctypes.c_void_p)]


class PfBranchSet(ctypes.Structure):
    _fields_ = [("nbr", ctypes.c_int), ("from_", ctypes.c_void_p), ("to", ctypes.c_void_p),
                ("yff_ri", ctypes.c_void_p), ("yft_ri", ctypes.c_void_p), ("vn_kv_from", ctypes.c_void_p),
                ("status", ctypes.c_void_p), ("sn_mva", ctypes.c_double)]


class PfSbusLayout(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("ngen", ctypes.c_int), ("nsgen", ctypes.c_int), ("nload", ctypes.c_int),
                ("gen_ptr", ctypes.c_void_p), ("gen_ids", ctypes.c_void_p), ("sgen_ptr", ctypes.c_void_p),
                ("sgen_ids", ctypes.c_void_p), ("load_ptr", ctypes.c_void_p), ("load_ids", ctypes.c_void_p)]


class PfServerGrid(ctypes.Structure):
    _fields_ = [("plan", ctypes.c_void_p), ("V0_ri", ctypes.c_void_p), ("Sbus_ri", ctypes.c_void_p),
                ("nbr", ctypes.c_int), ("case_ptr", ctypes.c_void_p), ("rows", ctypes.c_void_p),
                ("cols", ctypes.c_void_p), ("vals_ri", ctypes.c_void_p), ("max_iter", ctypes.c_int),
                ("tol", ctypes.c_double)]


#: exported symbols, as declared in include/lightsim2grid_b200.h
SYMBOLS = ("pf_last_error", "pf_plan_create", "pf_plan_destroy", "pf_plan_info_get", "pf_set_ybus_values",
           "pf_solve", "pf_get_J", "pf_batch_n1", "pf_n1_prepare", "pf_batch_ts", "pf_batch_device", "pf_timers",
           "pf_host_jacobian_pattern", "pf_host_schedule_solve", "pf_batch_device_phase_cycles",
           "pf_batch_device_phase_trace", "pf_batch_device_noalloc", "pf_batch_device_scratch",
           "pf_scratch_bytes", "pf_multi_create", "pf_multi_launch", "pf_multi_info", "pf_multi_destroy",
           "pf_flows_device", "pf_flows_host", "pf_ybus_positions", "pf_assemble_ybus_device",
           "pf_set_ybus_values_device", "pf_assemble_sbus_device", "pf_dc_plan_create", "pf_server_create",
           "pf_server_submit", "pf_server_poll", "pf_server_state", "pf_server_destroy", "pf_fdpf_plan_create", "pf_n1_order",
           "pf_server_configure", "pf_server_device_loop", "pf_server_latency_split")


def load(path=None):
    """Load the native library (raises if it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB
    if not os.path.exists(p):
        raise ImportError("lightsim2grid_b200: native library {} is missing; run "
                          "`python -m lightsim2grid_b200.build`".format(p))
    lib = ctypes.CDLL(p)
    lib.pf_last_error.restype = ctypes.c_char_p
    lib.pf_last_error.argtypes = []
    lib.pf_plan_create.restype = ctypes.c_int
    lib.pf_plan_create.argtypes = [ctypes.c_int, i32p, i32p, f64p, f64p, f64p, i32p, ctypes.c_int, f64p, i32p,
                                   ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(PfOptions),
                                   ctypes.POINTER(ctypes.c_void_p)]
    lib.pf_plan_destroy.restype = None
    lib.pf_plan_destroy.argtypes = [ctypes.c_void_p]
    lib.pf_plan_info_get.restype = ctypes.c_int
    lib.pf_plan_info_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfPlanInfo)]
    lib.pf_set_ybus_values.restype = ctypes.c_int
    lib.pf_set_ybus_values.argtypes = [ctypes.c_void_p, f64p]
    lib.pf_solve.restype = ctypes.c_int
    lib.pf_solve.argtypes = [ctypes.c_void_p, f64p, f64p, ctypes.c_int, ctypes.c_double, f64p, i32p, i32p, i32p]
    lib.pf_get_J.restype = ctypes.c_int
    lib.pf_get_J.argtypes = [ctypes.c_void_p, i32p, i32p, i32p, f64p]
    lib.pf_batch_n1.restype = ctypes.c_int
    lib.pf_batch_n1.argtypes = [ctypes.c_void_p, ctypes.c_int, i32p, i32p, i32p, f64p, f64p, f64p, ctypes.c_int,
                                ctypes.c_double, f64p, i32p, i32p, i32p]
    lib.pf_n1_prepare.restype = ctypes.c_int
    lib.pf_n1_prepare.argtypes = [ctypes.c_void_p, ctypes.c_int, i32p, i32p, i32p, f64p, i32p, i32p, i32p, f64p,
                                  ctypes.c_int]
    lib.pf_batch_ts.restype = ctypes.c_int
    lib.pf_batch_ts.argtypes = [ctypes.c_void_p, ctypes.c_int, f64p, f64p, ctypes.c_int, ctypes.c_int,
                                ctypes.c_double, f64p, i32p, i32p, i32p, i32p]
    lib.pf_batch_device.restype = ctypes.c_int
    lib.pf_batch_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfDeviceBatch), ctypes.c_void_p]
    lib.pf_batch_device_phase_cycles.restype = ctypes.c_int
    lib.pf_batch_device_phase_cycles.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfDeviceBatch), ctypes.c_void_p, f64p]
    lib.pf_batch_device_phase_trace.restype = ctypes.c_int
    lib.pf_batch_device_phase_trace.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfDeviceBatch), ctypes.c_void_p,
                                                f64p, ctypes.c_int]
    lib.pf_batch_device_noalloc.restype = ctypes.c_int
    lib.pf_batch_device_noalloc.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfDeviceBatch), ctypes.c_void_p]
    lib.pf_batch_device_scratch.restype = ctypes.c_int
    lib.pf_batch_device_scratch.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfDeviceBatch), ctypes.c_void_p,
                                            ctypes.c_longlong, ctypes.c_void_p]
    lib.pf_scratch_bytes.restype = ctypes.c_longlong
    lib.pf_scratch_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.pf_multi_create.restype = ctypes.c_int
    lib.pf_multi_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(PfDeviceBatch), ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p)]
    lib.pf_multi_launch.restype = ctypes.c_int
    lib.pf_multi_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.pf_multi_info.restype = ctypes.c_int
    lib.pf_multi_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    lib.pf_flows_device.restype = ctypes.c_int
    lib.pf_flows_device.argtypes = [ctypes.POINTER(PfBranchSet), ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.pf_flows_host.restype = ctypes.c_int
    lib.pf_flows_host.argtypes = [ctypes.POINTER(PfBranchSet), ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.pf_server_create.restype = ctypes.c_int
    lib.pf_server_create.argtypes = [ctypes.POINTER(PfServerGrid), ctypes.c_int, ctypes.c_longlong, ctypes.c_int,
                                     ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.pf_server_submit.restype = ctypes.c_int
    lib.pf_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.pf_server_poll.restype = ctypes.c_int
    lib.pf_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    lib.pf_server_configure.restype = ctypes.c_int
    lib.pf_server_configure.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.pf_server_device_loop.restype = ctypes.c_int
    lib.pf_server_device_loop.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.pf_server_state.restype = ctypes.c_int
    lib.pf_server_state.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.pf_server_latency_split.restype = ctypes.c_int
    lib.pf_server_latency_split.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    lib.pf_server_destroy.restype = None
    lib.pf_server_destroy.argtypes = [ctypes.c_void_p]
    lib.pf_dc_plan_create.restype = ctypes.c_int
    lib.pf_dc_plan_create.argtypes = [ctypes.c_int, i32p, i32p, f64p, i32p, ctypes.c_int, i32p, ctypes.c_int, i32p,
                                      ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    lib.pf_n1_order.restype = ctypes.c_int
    lib.pf_n1_order.argtypes = [ctypes.c_void_p, ctypes.c_int, i32p, i32p, f64p, f64p, i32p]
    lib.pf_fdpf_plan_create.restype = ctypes.c_int
    lib.pf_fdpf_plan_create.argtypes = [ctypes.c_int, i32p, i32p, f64p, i32p, i32p, f64p, i32p, i32p, f64p, i32p,
                                        ctypes.c_int, f64p, i32p, ctypes.c_int, i32p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_void_p)]
    lib.pf_ybus_positions.restype = ctypes.c_int
    lib.pf_ybus_positions.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
    lib.pf_assemble_ybus_device.restype = ctypes.c_int
    lib.pf_assemble_ybus_device.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 8
    lib.pf_set_ybus_values_device.restype = ctypes.c_int
    lib.pf_set_ybus_values_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.pf_assemble_sbus_device.restype = ctypes.c_int
    lib.pf_assemble_sbus_device.argtypes = [ctypes.POINTER(PfSbusLayout), ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                            ctypes.c_void_p, ctypes.c_void_p]
    lib.pf_multi_destroy.restype = None
    lib.pf_multi_destroy.argtypes = [ctypes.c_void_p]
    lib.pf_timers.restype = ctypes.c_int
    lib.pf_timers.argtypes = [ctypes.c_void_p, f64p, ctypes.c_int]
    lib.pf_host_jacobian_pattern.restype = ctypes.c_int
    lib.pf_host_jacobian_pattern.argtypes = [ctypes.c_int, i32p, i32p, f64p, i32p, ctypes.c_int, f64p, i32p,
                                             ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int, i32p, i32p, i32p]
    lib.pf_host_schedule_solve.restype = ctypes.c_int
    lib.pf_host_schedule_solve.argtypes = [ctypes.c_int, i32p, i32p, f64p, f64p, f64p, i32p, ctypes.c_int, f64p,
                                           i32p, ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int, f64p, f64p,
                                           ctypes.POINTER(PfPlanInfo)]
    if path is None:
        _lib = lib
    return lib


def last_error(lib=None):
    lib = lib or load()
    msg = lib.pf_last_error()
    return msg.decode() if msg else ""


def check(rc, what, lib=None):
    if rc != 0:
        raise RuntimeError("{} failed (status {}): {}".format(what, rc, last_error(lib)))


def as_i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def as_c128(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


def as_f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def ptr(a, t):
    return a.ctypes.data_as(t)


def cptr(a):
    """Pointer to a complex128 array as interleaved doubles."""
    return a.view(np.float64).ctypes.data_as(f64p)
