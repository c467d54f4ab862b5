"""Plan-based Python API over the C ABI (include/astroflow_dd.h).

A Plan holds the delay tables and the device workspace for one chunk geometry
(header, DM plan, band, RFI settings) and dedisperses any number of chunks of
that geometry.  Device buffers are torch tensors; torch is used for memory and
streams only, every sample is computed by the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib

_ALGOS = {"subband": _lib.ALGO_SUBBAND, "brute": _lib.ALGO_BRUTE}
_ZDM = {"callsite": _lib.ZDM_CALLSITE, "range": _lib.ZDM_RANGE, "range_ref": _lib.ZDM_RANGE_REF}
_TABLES = {"reference": _lib.TABLE_REFERENCE, "fp64": _lib.TABLE_FP64, "ieee": _lib.TABLE_IEEE}
_FREQ = {"header": _lib.FREQ_HEADER, "fil": _lib.FREQ_FIL}
_NP = {8: np.uint8, 16: np.uint16, 32: np.uint32}


@dataclass
class IqrmParams:
    """IQRM settings (the reference's iqrmconfig, include/rfi.h:12-39)."""
    mode: int = 0
    radius_frac: float = 0.10
    nsigma: float = 3.0
    geofactor: float = 1.5
    win_sec: float = 5.0
    hop_sec: float = 2.5
    include_tail: bool = True


@dataclass
class RfiParams:
    """RFI stage switches (the reference's rficonfig, include/rfi.h:41-57)."""
    use_mask: bool = False
    use_zero_dm: bool = False
    use_iqrm: bool = False
    iqrm: IqrmParams = field(default_factory=IqrmParams)


def _torch():
    import torch
    return torch


def _tdtype(bits: int):
    torch = _torch()
    return {8: torch.uint8, 16: torch.uint16, 32: torch.uint32, 64: torch.uint64}[bits]


class _FfiArgs:
    pass


def _ffi_args(header, dm_low, dm_high, freq_start, freq_end, dm_step, time_downsample, t_sample,
              algorithm, subband_width, ndm0, zero_dm_mode, table_mode, freq_mode, freq_table,
              rfi, bad_channels) -> _FfiArgs:
    """The C structs of dd_plan_create / dd_stream_open (kept alive by the caller)."""
    g = (lambda k: header[k]) if isinstance(header, dict) else (lambda k: getattr(header, k))
    a = _FfiArgs()
    a.nbits = int(g("nbits"))
    a.nchans = int(g("nchans"))
    a.h = _lib.Header(float(g("mjd")) if _has(header, "mjd") else 0.0, float(g("tsamp")),
                      float(g("fch1")), float(g("foff")), a.nbits, a.nchans, int(g("ndata")))
    a.freq_table = None if freq_table is None else np.ascontiguousarray(freq_table, np.float64)
    a.p = _lib.PlanParams(dm_low, dm_high, dm_step, freq_start, freq_end, int(time_downsample),
                          t_sample, _ALGOS[algorithm], int(subband_width), int(ndm0),
                          _ZDM[zero_dm_mode], _TABLES[table_mode], _FREQ[freq_mode],
                          None if a.freq_table is None else a.freq_table.ctypes.data)
    r = rfi or RfiParams()
    q = r.iqrm
    a.r = _lib.RfiConfig(int(r.use_mask), int(r.use_zero_dm), int(r.use_iqrm),
                         _lib.IqrmConfig(int(q.mode), q.radius_frac, q.nsigma, q.geofactor,
                                         q.win_sec, q.hop_sec, int(bool(q.include_tail))))
    a.bad = np.ascontiguousarray(list(bad_channels or []), np.int32)
    return a


class Plan:
    """One dedispersion geometry on one GPU.

    header: mapping/object with tsamp, fch1, foff, nbits, nchans, ndata (ascending
    frequency order, foff > 0).  algorithm "subband" follows the reference GPU
    path (src/core/dedispered.cu:988-1304), "brute" its CPU path
    (include/cpucal.hpp:75-201).
    """

    def __init__(self, header, dm_low: float, dm_high: float, freq_start: float,
                 freq_end: float, dm_step: float = 1.0, time_downsample: int = 1,
                 t_sample: float = 0.5, algorithm: str = "subband", subband_width: int = 32,
                 ndm0: int = 32, zero_dm_mode: str = "callsite", table_mode: str = "reference",
                 freq_mode: str = "header", freq_table: Optional[np.ndarray] = None,
                 rfi: Optional[RfiParams] = None, bad_channels: Optional[Sequence[int]] = None,
                 device: int = 0):
        L = _lib.load()
        a = _ffi_args(header, dm_low, dm_high, freq_start, freq_end, dm_step, time_downsample,
                      t_sample, algorithm, subband_width, ndm0, zero_dm_mode, table_mode,
                      freq_mode, freq_table, rfi, bad_channels)
        self.nbits, self.nchans, self.device = a.nbits, a.nchans, int(device)
        self._keep = a
        self._h = ctypes.c_void_p()
        _lib.check(L.dd_plan_create(ctypes.byref(a.h), ctypes.byref(a.p), ctypes.byref(a.r),
                                    a.bad.ctypes.data if a.bad.size else None, int(a.bad.size),
                                    self.device, ctypes.byref(self._h)))
        info = _lib.PlanInfo()
        _lib.check(L.dd_plan_get_info(self._h, ctypes.byref(info)))
        self.info = {n: getattr(info, n) for n, _ in _lib.PlanInfo._fields_}
        self.algorithm = algorithm
        self.out_shape = (int(self.info["dm_steps"]), int(self.info["out_cols"]))
        self.out_bits = 64 if self.nbits == 32 else 32
        self.in_shape = (int(self.info["nsamp_in"]), self.nchans)

    # ------------------------------------------------------------------ tables
    def tables(self):
        """(delay, residual) int32 arrays; residual is None for brute force."""
        i = self.info
        d = np.zeros((int(i["delay_rows"]), int(i["delay_cols"])), np.int32)
        r = None
        if self.algorithm == "subband":
            r = np.zeros((int(i["dm_steps"]), int(i["nsb"])), np.int32)
        _lib.check(_lib.load().dd_plan_get_tables(self._h, d.ctypes.data,
                                                  None if r is None else r.ctypes.data))
        return d, r

    def set_delay_table(self, delay: np.ndarray) -> None:
        delay = np.ascontiguousarray(delay, np.int32)
        if delay.shape != (int(self.info["delay_rows"]), int(self.info["delay_cols"])):
            raise ValueError(f"delay table must have shape {self.info['delay_rows'], self.info['delay_cols']}")
        _lib.check(_lib.load().dd_plan_set_delay_table(self._h, delay.ctypes.data))

    # ------------------------------------------------------------------ running
    def empty_output(self):
        torch = _torch()
        return torch.empty(self.out_shape, dtype=_tdtype(self.out_bits),
                           device=f"cuda:{self.device}")

    def run(self, x, out=None, stream=None, iqrm_masks=None, iqrm_bounds=None, prepped=None):
        """Dedisperse a device tensor x ([nsamp, nchans] or flat, uint8/16/32) into
        out ([dm_steps, out_cols] uint32, or uint64 for 32-bit input)."""
        torch = _torch()
        if not x.is_cuda or not x.is_contiguous():
            raise ValueError("input must be a contiguous CUDA tensor")
        if x.element_size() * 8 != self.nbits:
            raise ValueError(f"input dtype must be uint{self.nbits}")
        if x.numel() < self.in_shape[0] * self.in_shape[1]:
            raise ValueError("input holds fewer than ndata * nchans samples")
        if out is None:
            out = self.empty_output()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        ptr = lambda t: None if t is None else t.data_ptr()
        _lib.check(_lib.load().dd_run_ex(self._h, x.data_ptr(), out.data_ptr(), ptr(iqrm_masks),
                                         ptr(iqrm_bounds), ptr(prepped),
                                         ctypes.c_void_p(stream.cuda_stream)))
        return out

    def autotune(self, x, out=None, reps: int = 2, stream=None) -> dict:
        """Choose the launch shape (time tile, staging depth) of the subband path
        by timing dd_run on this chunk (dd_plan_autotune); results are unchanged."""
        torch = _torch()
        if out is None:
            out = self.empty_output()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        rep = _lib.TuneReport()
        L = _lib.load()
        _lib.check(L.dd_plan_autotune(self._h, x.data_ptr(), out.data_ptr(), int(reps),
                                      ctypes.c_void_p(stream.cuda_stream), ctypes.byref(rep)))
        info = _lib.PlanInfo()
        _lib.check(L.dd_plan_get_info(self._h, ctypes.byref(info)))
        self.info = {n: getattr(info, n) for n, _ in _lib.PlanInfo._fields_}
        return {n: getattr(rep, n) for n, _ in _lib.TuneReport._fields_ if n != "pad"}

    def run_profiled(self, x, out=None, stream=None) -> dict:
        """Run once and return the device-time breakdown (ms) and launch counts."""
        torch = _torch()
        if out is None:
            out = self.empty_output()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        st = _lib.RunStats()
        _lib.check(_lib.load().dd_run_profiled(self._h, x.data_ptr(), out.data_ptr(),
                                               ctypes.c_void_p(stream.cuda_stream),
                                               ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in _lib.RunStats._fields_}

    def run_host(self, x: np.ndarray, out: Optional[np.ndarray] = None, stream=None):
        """Dedisperse a host array through dd_run_host (copies inside the call)."""
        x = np.ascontiguousarray(x)
        if x.dtype != _NP[self.nbits]:
            raise ValueError(f"input dtype must be uint{self.nbits}")
        if x.size < self.in_shape[0] * self.in_shape[1]:
            raise ValueError("input holds fewer than ndata * nchans samples")
        if out is None:
            out = np.empty(self.out_shape, np.uint64 if self.out_bits == 64 else np.uint32)
        h = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        _lib.check(_lib.load().dd_run_host(self._h, x.ctypes.data, out.ctypes.data, h))
        return out

    def run_host_async(self, x: np.ndarray, out: np.ndarray, stream=None):
        """Queue a run of a host array through dd_run_host_async and return at once:
        `out` holds the result after run_host_join(stream, sync=True) (or once a
        stream joined with run_host_join(stream) has reached that point).  Chunks
        queued one after another overlap one chunk's output copy with the next
        one's input copy; both arrays should be in pinned memory and stay alive
        until then."""
        if x.dtype != _NP[self.nbits] or not x.flags.c_contiguous:
            raise ValueError(f"input must be a C-contiguous uint{self.nbits} array")
        if x.size < self.in_shape[0] * self.in_shape[1]:
            raise ValueError("input holds fewer than ndata * nchans samples")
        want = np.uint64 if self.out_bits == 64 else np.uint32
        if out.dtype != want or out.shape != self.out_shape or not out.flags.c_contiguous:
            raise ValueError(f"output must be a C-contiguous {want.__name__} array of shape {self.out_shape}")
        h = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        _lib.check(_lib.load().dd_run_host_async(self._h, x.ctypes.data, out.ctypes.data, h))
        return out

    def run_host_join(self, stream=None, sync: bool = False):
        """Make `stream` wait for the output copies of the queued run_host_async
        calls; with sync=True also wait on the host and report device errors."""
        h = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        _lib.check(_lib.load().dd_run_host_join(self._h, h, 1 if sync else 0))

    @property
    def closed(self) -> bool:
        return not (getattr(self, "_h", None) and self._h.value)

    def close(self, stream=None) -> None:
        """Release the plan.  With `stream` (the CUDA stream all of the plan's work
        was issued on) its memory is released stream-ordered, without waiting for
        the rest of the device."""
        if getattr(self, "_h", None) and self._h.value:
            if stream is None:
                _lib.load().dd_plan_destroy(self._h)
            else:
                _lib.load().dd_plan_destroy_async(self._h, ctypes.c_void_p(stream.cuda_stream))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MultiPlan:
    """Several DM ranges over one chunk with one upload: astroflow searches a list
    of (DM range, time downsampling) entries by one plain call per entry, each
    re-uploading the chunk (python/astroflow/search.py:519-534, 719-731); here the
    chunk stays resident and one Plan per range runs on it back to back.  Each
    range's output equals the plain call for that range.

    ranges: (dm_low, dm_high, dm_step, time_downsample) per entry; the other
    arguments are shared by every range (see Plan)."""

    def __init__(self, header, ranges, freq_start: float, freq_end: float, **plan_kwargs):
        if not ranges:
            raise ValueError("a multi-range plan needs at least one range")
        self.plans = []
        try:
            for lo, hi, step, ds in ranges:
                self.plans.append(Plan(header, lo, hi, freq_start, freq_end, step, ds,
                                       **plan_kwargs))
        except Exception:
            self.close()
            raise
        self.in_shape = self.plans[0].in_shape
        self.nbits = self.plans[0].nbits
        self.device = self.plans[0].device

    @property
    def workspace_bytes(self) -> int:
        return int(sum(p.info["workspace_bytes"] for p in self.plans))

    @property
    def output_bytes(self) -> int:
        return int(sum(p.out_shape[0] * p.out_shape[1] * p.out_bits // 8 for p in self.plans))

    def empty_outputs(self):
        return [p.empty_output() for p in self.plans]

    def run(self, x, outs=None, stream=None):
        """x: the resident chunk (device tensor); returns one output per range."""
        if outs is None:
            outs = self.empty_outputs()
        for p, o in zip(self.plans, outs):
            p.run(x, o, stream)
        return outs

    def close(self) -> None:
        for p in self.plans:
            p.close()
        self.plans = []


class Batch:
    """Many chunks of different geometries in one run (dd_batch_*): each plan's
    RFI/layout kernels, then the dedispersion sums of all plans batched (one
    launch per tile, stage and kernel variant over every plan, or with
    persistent=True one persistent launch), captured in a CUDA graph and
    replayed while the same buffers are passed.  Results equal Plan.run of each
    plan on its chunk."""

    def __init__(self, plans: Sequence[Plan], use_graph: bool = True, persistent: bool = False):
        if not plans:
            raise ValueError("a batch needs at least one plan")
        self.plans = list(plans)
        arr = (ctypes.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        self._h = ctypes.c_void_p()
        flags = (_lib.BATCH_GRAPH if use_graph else 0) | (_lib.BATCH_PERSISTENT if persistent else 0)
        _lib.check(_lib.load().dd_batch_create(arr, len(self.plans), flags, ctypes.byref(self._h)))

    def empty_outputs(self):
        return [p.empty_output() for p in self.plans]

    def run(self, inputs, outputs=None, stream=None):
        """inputs/outputs: one device tensor per plan (as for Plan.run)."""
        torch = _torch()
        if len(inputs) != len(self.plans):
            raise ValueError(f"expected {len(self.plans)} inputs")
        if outputs is None:
            outputs = self.empty_outputs()
        for p, x, o in zip(self.plans, inputs, outputs):
            if not x.is_cuda or not x.is_contiguous() or x.element_size() * 8 != p.nbits:
                raise ValueError(f"input must be a contiguous CUDA tensor of uint{p.nbits}")
            if x.numel() < p.in_shape[0] * p.in_shape[1]:
                raise ValueError("input holds fewer than ndata * nchans samples")
            if tuple(o.shape) != p.out_shape or not o.is_cuda:
                raise ValueError(f"output must be a CUDA tensor of shape {p.out_shape}")
        if stream is None:
            stream = torch.cuda.current_stream(self.plans[0].device)
        ins = (ctypes.c_void_p * len(inputs))(*[x.data_ptr() for x in inputs])
        outs = (ctypes.c_void_p * len(outputs))(*[o.data_ptr() for o in outputs])
        _lib.check(_lib.load().dd_batch_run(self._h, ins, outs, ctypes.c_void_p(stream.cuda_stream)))
        return outputs

    def status(self) -> None:
        """Wait for the batch's work; raise if a bounded device wait gave up."""
        _lib.check(_lib.load().dd_batch_status(self._h))

    @property
    def info(self) -> dict:
        i = _lib.BatchInfo()
        _lib.check(_lib.load().dd_batch_get_info(self._h, ctypes.byref(i)))
        return {n: getattr(i, n) for n, _ in _lib.BatchInfo._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().dd_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Stream:
    """A beam dedispersed chunk by chunk (dd_stream_*): the beam's last `tail`
    samples stay on the device and every push is the plain subband call on
    [tail | chunk], returning its first chunk/time_downsample columns.  header
    describes one chunk (ndata = samples per push)."""

    def __init__(self, header, dm_low: float, dm_high: float, freq_start: float,
                 freq_end: float, dm_step: float = 1.0, time_downsample: int = 1,
                 subband_width: int = 32, ndm0: int = 32, zero_dm_mode: str = "callsite",
                 table_mode: str = "reference", freq_mode: str = "header",
                 freq_table: Optional[np.ndarray] = None, rfi: Optional[RfiParams] = None,
                 bad_channels: Optional[Sequence[int]] = None, device: int = 0):
        L = _lib.load()
        a = _ffi_args(header, dm_low, dm_high, freq_start, freq_end, dm_step, time_downsample,
                      0.5, "subband", subband_width, ndm0, zero_dm_mode, table_mode, freq_mode,
                      freq_table, rfi, bad_channels)
        self.nbits, self.nchans, self.device = a.nbits, a.nchans, int(device)
        self._keep = a
        self._h = ctypes.c_void_p()
        _lib.check(L.dd_stream_open(ctypes.byref(a.h), ctypes.byref(a.p), ctypes.byref(a.r),
                                    a.bad.ctypes.data if a.bad.size else None, int(a.bad.size),
                                    self.device, ctypes.byref(self._h)))
        self.out_shape = (int(self.info["dm_steps"]), int(self.info["out_cols"]))
        self.chunk_shape = (int(self.info["chunk_samples"]), self.nchans)

    @property
    def info(self) -> dict:
        i = _lib.StreamInfo()
        _lib.check(_lib.load().dd_stream_get_info(self._h, ctypes.byref(i)))
        return {n: getattr(i, n) for n, _ in _lib.StreamInfo._fields_}

    def empty_output(self):
        torch = _torch()
        return torch.empty(self.out_shape, dtype=_tdtype(64 if self.nbits == 32 else 32),
                           device=f"cuda:{self.device}")

    def push(self, chunk, out=None, stream=None):
        """chunk: contiguous CUDA tensor of chunk_shape samples; returns out."""
        torch = _torch()
        if not chunk.is_cuda or not chunk.is_contiguous() or chunk.element_size() * 8 != self.nbits:
            raise ValueError(f"chunk must be a contiguous CUDA tensor of uint{self.nbits}")
        if chunk.numel() != self.chunk_shape[0] * self.chunk_shape[1]:
            raise ValueError(f"chunk must hold {self.chunk_shape} samples")
        if out is None:
            out = self.empty_output()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        _lib.check(_lib.load().dd_stream_push(self._h, chunk.data_ptr(), out.data_ptr(),
                                              ctypes.c_void_p(stream.cuda_stream)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().dd_stream_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def single_dm_spectrum(x, header, tstart: float, tend: float, dm: float, freq_start: float,
                       freq_end: float, freq_mode: str = "header",
                       freq_table: Optional[np.ndarray] = None, rfi: Optional[RfiParams] = None,
                       bad_channels: Optional[Sequence[int]] = None, masked_rows: bool = False,
                       stream=None):
    """Dedispersed spectrum at one DM over [tstart, tend) (dd_single_dm_run): the
    selected channels, each shifted by its delay.  x: device tensor [ndata, nchans].
    Returns (spectrum [ntimes, nsel] device tensor, geometry dict, the RFI-processed
    rows [rfi_len, nchans] or None)."""
    torch = _torch()
    L = _lib.load()
    a = _ffi_args(header, 0.0, 1.0, freq_start, freq_end, 1.0, 1, 0.5, "subband", 32, 32,
                  "callsite", "reference", freq_mode, freq_table, rfi, bad_channels)
    q = _lib.SingleDmParams(tstart, tend, dm, freq_start, freq_end, _FREQ[freq_mode],
                            None if a.freq_table is None else a.freq_table.ctypes.data)
    info = _lib.SingleDmInfo()
    _lib.check(L.dd_single_dm_geometry(ctypes.byref(a.h), ctypes.byref(q), ctypes.byref(info)))
    g = {n: getattr(info, n) for n, _ in _lib.SingleDmInfo._fields_}
    if not x.is_cuda or not x.is_contiguous() or x.element_size() * 8 != a.nbits:
        raise ValueError(f"x must be a contiguous CUDA tensor of uint{a.nbits}")
    if x.numel() < int(a.h.ndata) * a.nchans:
        raise ValueError("x holds fewer than ndata * nchans samples")
    dt = _tdtype(a.nbits)
    out = torch.empty((g["ntimes"], g["nchans"]), dtype=dt, device=x.device)
    rows = torch.empty((g["rfi_len"], a.nchans), dtype=dt, device=x.device) if masked_rows else None
    if stream is None:
        stream = torch.cuda.current_stream(x.device)
    _lib.check(L.dd_single_dm_run(ctypes.byref(a.h), ctypes.byref(q), ctypes.byref(a.r),
                                  a.bad.ctypes.data if a.bad.size else None, int(a.bad.size),
                                  x.data_ptr(), out.data_ptr(),
                                  None if rows is None else rows.data_ptr(),
                                  ctypes.c_void_p(stream.cuda_stream)))
    return out, g, rows


def iqrm_masks_noalloc(x, nchans: int, chan_start: int, chan_end: int, tsamp: float,
                       iqrm: IqrmParams, masks, bounds, stream=None) -> int:
    """IQRM window masks through dd_iqrm_masks_noalloc: no device memory is
    allocated by the library; `masks` ([max_windows, nchans] uint8) and `bounds`
    ([max_windows, 2] int32/uint32) are caller-owned device tensors on the current
    device.  For callers that cannot allocate while they run (deadline-bound
    real-time loops, frameworks that own the GPU's memory).  Calls share one
    static scratch array per GPU, so their GPU work must not overlap.  Returns
    the number of windows."""
    torch = _torch()
    nchans, chan_start, chan_end = int(nchans), int(chan_start), int(chan_end)
    if nchans < 1:
        raise ValueError("nchans must be >= 1")
    if x.dtype not in (torch.uint8, torch.uint16, torch.uint32, torch.int16, torch.int32):
        raise ValueError("x must hold 8-, 16- or 32-bit samples")
    if not x.is_contiguous() or x.numel() == 0 or x.numel() % nchans:
        raise ValueError("x must be a non-empty contiguous tensor of whole [nsamp, nchans] rows")
    if masks.dtype != torch.uint8 or masks.dim() != 2 or masks.shape[1] != nchans \
            or not masks.is_contiguous():
        raise ValueError("masks must be a contiguous uint8 tensor of shape [max_windows, nchans]")
    if bounds.dtype not in (torch.int32, torch.uint32) or bounds.dim() != 2 \
            or bounds.shape[1] != 2 or bounds.shape[0] < masks.shape[0] or not bounds.is_contiguous():
        raise ValueError("bounds must be a contiguous int32 tensor of shape [>= max_windows, 2]")
    if not (0 <= chan_start < chan_end <= nchans):
        raise ValueError("channel range must satisfy 0 <= chan_start < chan_end <= nchans")
    for name, t in (("x", x), ("masks", masks), ("bounds", bounds)):
        if not t.is_cuda or t.device.index != torch.cuda.current_device():
            raise ValueError(f"{name} must be on the current CUDA device")
    if stream is None:
        stream = torch.cuda.current_stream()
    n = ctypes.c_int32()
    q = _lib.IqrmConfig(int(iqrm.mode), iqrm.radius_frac, iqrm.nsigma, iqrm.geofactor,
                        iqrm.win_sec, iqrm.hop_sec, int(bool(iqrm.include_tail)))
    _lib.check(_lib.load().dd_iqrm_masks_noalloc(
        x.data_ptr(), x.element_size() * 8, x.numel() // nchans, nchans, chan_start, chan_end,
        tsamp, ctypes.byref(q), masks.data_ptr(), bounds.data_ptr(), masks.shape[0],
        ctypes.byref(n), ctypes.c_void_p(stream.cuda_stream)))
    return n.value


def brute_delay_table(freq, chan_start: int, chan_end: int, ref_channel: int, dm_low: float,
                      dm_step: float, dm_steps: int, tsamp: float, table_mode: str = "reference"):
    """The brute-force delay table (include/cpucal.hpp:119-132) computed on the host
    without a plan or a GPU (dd_brute_delay_table): an int32 array
    [dm_steps, chan_end - chan_start] and the number of entries that differ from
    the FP64 evaluation."""
    f = np.ascontiguousarray(freq, dtype=np.float64)
    if not (0 <= chan_start < chan_end <= f.size and 0 <= ref_channel < f.size):
        raise ValueError("channel range or reference channel outside the frequency table")
    out = np.zeros((int(dm_steps), chan_end - chan_start), np.int32)
    mism = ctypes.c_int64()
    _lib.check(_lib.load().dd_brute_delay_table(
        f.ctypes.data, int(chan_start), int(chan_end), int(ref_channel), float(dm_low),
        float(dm_step), int(dm_steps), float(tsamp), _TABLES[table_mode], out.ctypes.data,
        ctypes.byref(mism)))
    return out, mism.value


def measure_int_add_rate(device: int = 0) -> float:
    """Sustained 32-bit integer additions per second on `device` (library probe)."""
    v = ctypes.c_double()
    _lib.check(_lib.load().dd_measure_int_add_rate(int(device), ctypes.byref(v)))
    return v.value


def _has(obj, k):
    return (k in obj) if isinstance(obj, dict) else hasattr(obj, k)
