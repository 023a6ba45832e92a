"""ctypes binding of libedlut_b200.so (the C ABI declared in include/edlut_b200.h).

The library is built in-tree (``edlut_b200/_lib/libedlut_b200.so``) by
:func:`edlut_b200.build.build`.  Loading fails loudly when it is missing: there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libedlut_b200.so")

EB_OK = 0
ERRORS = {-1: "EB_ERR_ARG", -2: "EB_ERR_CUDA", -3: "EB_ERR_STATE", -4: "EB_ERR_OVERFLOW",
          -5: "EB_ERR_PARSE", -6: "EB_ERR_UNSUPPORTED", -7: "EB_ERR_NOMEM", -8: "EB_ERR_NUMERIC"}
KINDS = {"InputSpikeNeuronModel": 0, "LIFTimeDrivenModel": 1, "AdExTimeDrivenModel": 2,
         "HHTimeDrivenModel": 3, "PoissonGeneratorDeviceVector": 4}
INTEGRATORS = {"Euler": 0, "RK2": 1, "RK4": 2, "BDF": 3}

c_i64p = ctypes.POINTER(ctypes.c_int64)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_f64p = ctypes.POINTER(ctypes.c_double)

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("eb_last_error", ctypes.c_char_p, []),
    ("eb_version", ctypes.c_char_p, []),
    ("eb_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("eb_ctx_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("eb_add_population", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_float, c_f32p, ctypes.c_int, c_i64p]),
    ("eb_add_stdp_rule", ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_float, ctypes.POINTER(ctypes.c_int)]),
    ("eb_set_connectivity", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, c_i64p, c_i64p, c_f32p, c_i32p,
                                            c_f32p, c_f32p, c_i32p]),
    ("eb_set_bucket_limit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    ("eb_set_wide_indegree", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("eb_set_barrier_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int]),
    ("eb_enable_conductances", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("eb_population_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    ("eb_finalize", ctypes.c_int, [ctypes.c_void_p, c_i64p]),
    ("eb_load_network_files", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p]),
    ("eb_inject_spikes", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, c_f32p, c_i64p]),
    ("eb_load_input_file", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    ("eb_run", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("eb_run_async", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("eb_sync", ctypes.c_int, [ctypes.c_void_p]),
    ("eb_set_graph_steps", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("eb_set_persistent", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("eb_set_timeline", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("eb_get_timeline", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]),
    ("eb_set_record_capacity", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("eb_get_spikes", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, c_i64p, c_i64p, c_i64p]),
    ("eb_step_time", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, c_f64p]),
    ("eb_get_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, c_f32p]),
    ("eb_set_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, c_f32p]),
    ("eb_set_trace", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]),
    ("eb_get_trace", ctypes.c_int, [ctypes.c_void_p, c_f32p]),
    ("eb_write_spikes", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]),
    ("eb_set_output", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("eb_set_monitor", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("eb_open_monitor", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64]),
    ("eb_close_monitor", ctypes.c_int, [ctypes.c_void_p]),
    ("eb_save_weights", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    ("eb_get_weights", ctypes.c_int, [ctypes.c_void_p, c_f32p]),
    ("eb_set_weights", ctypes.c_int, [ctypes.c_void_p, c_f32p]),
    ("eb_get_counters", ctypes.c_int, [ctypes.c_void_p, c_i64p, c_i64p, c_i64p]),
    ("eb_device_bytes", ctypes.c_int, [ctypes.c_void_p, c_i64p]),
    ("eb_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("eb_prestage", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("eb_set_profile", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("eb_get_profile", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), c_i64p, c_f64p]),
    ("eb_launch_count", ctypes.c_int, [ctypes.c_void_p, c_i64p]),
    ("eb_fold_arrivals", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    ("eb_fold_arrivals_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p]),
    ("eb_get_population_events", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_i64p]),
    ("eb_set_random_seed", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    ("eb_set_poisson_rates", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, c_f32p]),
    ("eb_snapshot", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("eb_restore", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    # batched sweep
    ("eb_sweep_create", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("eb_sweep_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("eb_sweep_set_network", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, c_f32p, ctypes.c_float, ctypes.c_float,
                                             ctypes.c_float, ctypes.c_float]),
    ("eb_sweep_set_inputs", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, c_f32p, c_i32p]),
    ("eb_sweep_build", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_float]),
    ("eb_sweep_reset", ctypes.c_int, [ctypes.c_void_p]),
    ("eb_sweep_configure", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("eb_sweep_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)]),
    ("eb_sweep_run", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("eb_sweep_run_async", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("eb_sweep_sync", ctypes.c_int, [ctypes.c_void_p]),
    ("eb_sweep_get_spikes", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, c_i64p, c_i32p,
                                            c_i32p]),
    ("eb_sweep_spike_counts", ctypes.c_int, [ctypes.c_void_p, c_i64p]),
    ("eb_sweep_get_synapses", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, c_i64p, c_i32p,
                                              c_i32p, c_f32p]),
    ("eb_sweep_get_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_f32p]),
    ("eb_sweep_info", ctypes.c_int, [ctypes.c_void_p, c_i64p, c_i64p, c_i64p, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("eb_sweep_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("eb_sweep_set_synapses", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, c_i32p, c_i32p,
                                              c_f32p]),
    ("eb_sweep_set_params", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_f32p]),
    ("eb_sweep_set_weights", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    ("eb_sweep_get_weights", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    ("eb_sweep_set_observed", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_i32p]),
    ("eb_sweep_get_trace", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    ("eb_sweep_set_checkpoints", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("eb_sweep_adjoint", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_int, c_f64p]),
]

_lib = None


class EdlutError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "EB_ERR"), code, msg))
        self.code = code


def load():
    """Load libedlut_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("edlut_b200 CUDA library not built: %s is missing "
                               "(run __graft_entry__.build() or python -m edlut_b200.build)" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(rc: int) -> None:
    if rc != EB_OK:
        raise EdlutError(rc, load().eb_last_error().decode())
