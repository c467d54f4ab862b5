"""ctypes binding of libastroflow_dd.so (declared in include/astroflow_dd.h).

The library is built in-tree by astroflow_b200/build.py.  Loading fails loudly
when it is missing: there is no CPU fallback for the dedispersion path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# ASTROFLOW_DD_LIB selects another build of the library (e.g. a tuning variant).
LIB_PATH = os.environ.get("ASTROFLOW_DD_LIB") or os.path.join(HERE, "libastroflow_dd.so")

DD_OK = 0
DD_ERR_INVALID = 1
DD_ERR_RUNTIME = 2
DD_ERR_CUDA = 3
DD_ERR_NOMEM = 4
DD_ERR_TIMEOUT = 5
DD_ERR_UNSUPPORTED = 6

ALGO_SUBBAND, ALGO_BRUTE = 0, 1
ZDM_CALLSITE, ZDM_RANGE, ZDM_RANGE_REF = 0, 1, 2
TABLE_REFERENCE, TABLE_FP64, TABLE_IEEE = 0, 1, 2
FREQ_HEADER, FREQ_FIL = 0, 1

# Every symbol include/astroflow_dd.h declares.
EXPORTS = ("dd_plan_create", "dd_plan_destroy", "dd_plan_destroy_async", "dd_plan_get_info",
           "dd_plan_get_tables", "dd_brute_delay_table",
           "dd_plan_set_delay_table", "dd_run", "dd_run_ex", "dd_run_host", "dd_run_host_async",
           "dd_run_host_join", "dd_run_profiled",
           "dd_measure_int_add_rate", "dd_iqrm_masks_noalloc", "dd_batch_create",
           "dd_batch_run", "dd_batch_status", "dd_batch_get_info", "dd_batch_destroy",
           "dd_stream_open", "dd_stream_push", "dd_stream_get_info", "dd_stream_plan",
           "dd_stream_close", "dd_single_dm_geometry", "dd_single_dm_run",
           "dd_images", "dd_fil_read_header", "dd_fil_read", "dd_ingest_host", "dd_launch_count",
           "dd_plan_autotune",
           "dd_last_error", "dd_abi_version")


class Header(ctypes.Structure):
    _fields_ = [("mjd", ctypes.c_double), ("tsamp", ctypes.c_double), ("fch1", ctypes.c_double),
                ("foff", ctypes.c_double), ("nbits", ctypes.c_int32), ("nchans", ctypes.c_int32),
                ("ndata", ctypes.c_int64)]


class IqrmConfig(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("radius_frac", ctypes.c_float),
                ("nsigma", ctypes.c_float), ("geofactor", ctypes.c_double),
                ("win_sec", ctypes.c_double), ("hop_sec", ctypes.c_double),
                ("include_tail", ctypes.c_int32)]


class RfiConfig(ctypes.Structure):
    _fields_ = [("use_mask", ctypes.c_int32), ("use_zero_dm", ctypes.c_int32),
                ("use_iqrm", ctypes.c_int32), ("iqrm", IqrmConfig)]


class PlanParams(ctypes.Structure):
    _fields_ = [("dm_low", ctypes.c_float), ("dm_high", ctypes.c_float),
                ("dm_step", ctypes.c_float), ("freq_start", ctypes.c_float),
                ("freq_end", ctypes.c_float), ("time_downsample", ctypes.c_int32),
                ("t_sample", ctypes.c_float), ("algorithm", ctypes.c_int32),
                ("subband_width", ctypes.c_int32), ("ndm0", ctypes.c_int32),
                ("zero_dm_mode", ctypes.c_int32), ("table_mode", ctypes.c_int32),
                ("freq_mode", ctypes.c_int32), ("freq_table", ctypes.c_void_p)]


class PlanInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "chan_start", "chan_end", "dm_steps", "nsamp_in", "nsamp_binned", "out_cols",
        "out_elem_bytes", "nsb", "ndm_nom", "max_delay", "max_residual", "nslices",
        "n_iqrm_windows", "workspace_bytes", "delay_rows", "delay_cols",
        "table_mismatch_fp64", "tile_samples")] + [("adds_per_run", ctypes.c_double),
                                                    ("subband_sum_copies", ctypes.c_int64)]


class BatchInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("nplans", "groups", "blocks", "sum_launches",
                                               "launches", "own_plans")] + \
               [(n, ctypes.c_int32) for n in ("graph", "persistent", "graph_captures", "pad")]


class StreamInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("dm_steps", "out_cols", "chunk_samples",
                                               "tail_samples", "pushed_samples",
                                               "workspace_bytes")] + \
               [("adds_per_push", ctypes.c_double)]


class SingleDmParams(ctypes.Structure):
    _fields_ = [("tstart", ctypes.c_float), ("tend", ctypes.c_float), ("dm", ctypes.c_float),
                ("freq_start", ctypes.c_float), ("freq_end", ctypes.c_float),
                ("freq_mode", ctypes.c_int32), ("freq_table", ctypes.c_void_p)]


class SingleDmInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("t_start", "ntimes", "chan_start", "nchans",
                                               "rfi_t0", "rfi_len")] + \
               [("tend", ctypes.c_float), ("freq_start", ctypes.c_float),
                ("freq_end", ctypes.c_float), ("pad", ctypes.c_int32)]


class TuneReport(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_int64), ("best_budget_bytes", ctypes.c_int64),
                ("best_tile_samples", ctypes.c_int64), ("best_stages", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("best_ms", ctypes.c_double),
                ("default_ms", ctypes.c_double)]


BATCH_GRAPH = 1
BATCH_PERSISTENT = 2


class RunStats(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_float), ("prep_ms", ctypes.c_float),
                ("stage1_ms", ctypes.c_float), ("stage2_ms", ctypes.c_float),
                ("launches", ctypes.c_int32), ("stage1_launches", ctypes.c_int32),
                ("stage2_launches", ctypes.c_int32)]


_lib = None


def load():
    """Load the library (once).  Raises RuntimeError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m astroflow_b200.build` "
            "(there is no CPU fallback for the dedispersion path)")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    L.dd_plan_create.argtypes = [ctypes.POINTER(Header), ctypes.POINTER(PlanParams),
                                 ctypes.POINTER(RfiConfig), P, ctypes.c_int32, ctypes.c_int32,
                                 ctypes.POINTER(ctypes.c_void_p)]
    L.dd_plan_destroy.argtypes = [P]
    L.dd_plan_get_info.argtypes = [P, ctypes.POINTER(PlanInfo)]
    L.dd_plan_get_tables.argtypes = [P, P, P]
    L.dd_brute_delay_table.argtypes = [P, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_int64,
                                       ctypes.c_double, ctypes.c_int32, P, P]
    L.dd_plan_set_delay_table.argtypes = [P, P]
    L.dd_run.argtypes = [P, P, P, P]
    L.dd_run_ex.argtypes = [P, P, P, P, P, P, P]
    L.dd_run_host.argtypes = [P, P, P, P]
    L.dd_run_host_async.argtypes = [P, P, P, P]
    L.dd_run_host_join.argtypes = [P, P, ctypes.c_int32]
    L.dd_run_profiled.argtypes = [P, P, P, P, ctypes.POINTER(RunStats)]
    L.dd_measure_int_add_rate.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
    L.dd_iqrm_masks_noalloc.argtypes = [P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                        ctypes.POINTER(IqrmConfig), P, P, ctypes.c_int32,
                                        ctypes.POINTER(ctypes.c_int32), P]
    L.dd_last_error.restype = ctypes.c_char_p
    L.dd_abi_version.restype = ctypes.c_int
    L.dd_batch_create.argtypes = [ctypes.POINTER(P), ctypes.c_int32, ctypes.c_int32,
                                  ctypes.POINTER(P)]
    L.dd_batch_run.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), P]
    L.dd_batch_status.argtypes = [P]
    L.dd_batch_get_info.argtypes = [P, ctypes.POINTER(BatchInfo)]
    L.dd_batch_destroy.argtypes = [P]
    L.dd_plan_destroy_async.argtypes = [P, P]
    L.dd_single_dm_geometry.argtypes = [ctypes.POINTER(Header), ctypes.POINTER(SingleDmParams),
                                        ctypes.POINTER(SingleDmInfo)]
    L.dd_single_dm_run.argtypes = [ctypes.POINTER(Header), ctypes.POINTER(SingleDmParams),
                                   ctypes.POINTER(RfiConfig), P, ctypes.c_int32, P, P, P, P]
    L.dd_launch_count.argtypes = [ctypes.POINTER(ctypes.c_int64)]
    L.dd_plan_autotune.argtypes = [P, P, P, ctypes.c_int32, P, ctypes.POINTER(TuneReport)]
    L.dd_images.argtypes = [P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, P, P,
                            ctypes.c_int32, P, P, P, P]
    L.dd_stream_open.argtypes = [ctypes.POINTER(Header), ctypes.POINTER(PlanParams),
                                 ctypes.POINTER(RfiConfig), P, ctypes.c_int32, ctypes.c_int32,
                                 ctypes.POINTER(P)]
    L.dd_stream_push.argtypes = [P, P, P, P]
    L.dd_stream_get_info.argtypes = [P, ctypes.POINTER(StreamInfo)]
    L.dd_stream_plan.argtypes = [P, ctypes.POINTER(P)]
    L.dd_stream_close.argtypes = [P]
    for name in EXPORTS:
        if name not in ("dd_last_error", "dd_abi_version"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def check(rc: int) -> None:
    """Map a status code to the exception the reference raises for it."""
    if rc == DD_OK:
        return
    msg = load().dd_last_error().decode(errors="replace")
    if rc == DD_ERR_INVALID:
        raise ValueError(msg)
    if rc == DD_ERR_NOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def launch_count() -> int:
    """Kernels the library has launched from the calling thread."""
    n = ctypes.c_int64()
    check(load().dd_launch_count(ctypes.byref(n)))
    return n.value
