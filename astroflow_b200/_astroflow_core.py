"""Drop-in replacement for astroflow's pybind11 module ``_astroflow_core`` on the
dedispersion path (src/bindpy/bindings.cpp:13-74, src/bindpy/pyapi.cpp).

Same names, constructors, argument order, defaults and exceptions as the bound
C++; the work runs in libastroflow_dd.so on the GPU:

  _dedisperse_spec(data, header, dm_low, dm_high, freq_start, freq_end, dm_step,
                   time_downsample, t_sample, target_id, mask_file, rficfg)
      -> DedispersedDataUint8                      (bindings.cpp:43-57, pyapi.cpp:284-309)
  _dedispered_fil(filename, dm_low, dm_high, freq_start, freq_end, dm_step,
                  time_downsample, t_sample, target=1, target_id=0,
                  maskfile="mask.txt", rficfg=RFIconfig())   (bindings.cpp:25-29, pyapi.cpp:6-51)
  Header, IQRMconfig, RFIconfig, DedispersedDataUint8, DedisperedData, Filterbank,
  Spectrum8/16/32

Keyword names of _dedisperse_spec are the ones the reference binds, which are
shifted by one position from the C++ parameters (the 6th positional argument is
freq_end although it is bound as ``dm_step``); callers pass them positionally
(python/astroflow/dedispered.py:59-72) and so does everything here.

Compile-time choices of the reference become module settings: the subband width
(AF_SUBBAND_SIZE_CH, default 32, dedispered.cu:29-31) and the zero-DM form
(the reference's call-site behaviour by default); both can be set through
ASTROFLOW_SUBBAND_WIDTH and ASTROFLOW_ZERO_DM_MODE ("callsite" or "range").
"""
from __future__ import annotations

import os
import re
import struct
import threading
from collections import OrderedDict
from contextlib import contextmanager
from typing import List, Optional, Tuple

import numpy as np

from . import ingest, postprocess
from .dedisp import IqrmParams, Plan, RfiParams

REF_FREQ_END = 1
REF_FREQ_START = 0
CPU_TARGET = 0
GPU_TARGET = 1

SUBBAND_WIDTH = int(os.environ.get("ASTROFLOW_SUBBAND_WIDTH", "32"))
NDM0 = 32
ZERO_DM_MODE = os.environ.get("ASTROFLOW_ZERO_DM_MODE", "callsite")


def _f32(v) -> float:
    return float(np.float32(v))


# ------------------------------------------------------------------ config types
class IQRMconfig:
    """include/rfi.h:12-39 and its binding (pyapi.cpp:242-254)."""

    def __init__(self, *args):
        if len(args) == 0:
            vals = (0, 0.10, 3.0, 1.5, 5.0, 2.5, True)
            self._set(vals, float_all=True)
        elif len(args) == 7:
            # init<int, float, float, float, float, float, bool>: every real is a float
            self._set(args, float_all=True)
        elif len(args) == 1:
            o = args[0]
            self._mode = int(o.mode)
            self._radius_frac = _f32(o.radius_frac)
            self._nsigma = _f32(o.nsigma)
            self._geofactor = float(o.geofactor)
            self._win_sec = float(o.win_sec)
            self._hop_sec = float(o.hop_sec)
            self._include_tail = bool(o.include_tail)
        else:
            raise TypeError("IQRMconfig(): expected (), (mode, radius_frac, nsigma, geofactor, "
                            "win_sec, hop_sec, include_tail) or (object)")

    def _set(self, v, float_all):
        self._mode = int(v[0])
        self._radius_frac = _f32(v[1])
        self._nsigma = _f32(v[2])
        self._geofactor = _f32(v[3])
        self._win_sec = _f32(v[4])
        self._hop_sec = _f32(v[5])
        self._include_tail = bool(v[6])

    mode = property(lambda s: s._mode)
    radius_frac = property(lambda s: s._radius_frac)
    nsigma = property(lambda s: s._nsigma)
    geofactor = property(lambda s: s._geofactor)
    win_sec = property(lambda s: s._win_sec)
    hop_sec = property(lambda s: s._hop_sec)
    include_tail = property(lambda s: s._include_tail)

    def params(self) -> IqrmParams:
        return IqrmParams(self._mode, self._radius_frac, self._nsigma, self._geofactor,
                          self._win_sec, self._hop_sec, self._include_tail)


class RFIconfig:
    """include/rfi.h:41-57 and its binding (pyapi.cpp:257-266)."""

    def __init__(self, *args):
        if len(args) == 0:
            self._use_mask = self._use_zero_dm = self._use_iqrm = False
            self._iqrm_cfg = IQRMconfig()
        elif len(args) == 4:
            self._use_mask, self._use_zero_dm, self._use_iqrm = (bool(a) for a in args[:3])
            cfg = args[3]
            self._iqrm_cfg = cfg if isinstance(cfg, IQRMconfig) else IQRMconfig(cfg)
        elif len(args) == 1:
            o = args[0]
            self._use_zero_dm = bool(o.use_zero_dm)
            self._use_mask = bool(o.use_mask)
            self._use_iqrm = bool(o.use_iqrm)
            self._iqrm_cfg = IQRMconfig(o.iqrm_cfg)
        else:
            raise TypeError("RFIconfig(): expected (), (use_mask, use_zero_dm, use_iqrm, "
                            "iqrm_cfg) or (object)")

    use_zero_dm = property(lambda s: s._use_zero_dm)
    use_mask = property(lambda s: s._use_mask)
    use_iqrm = property(lambda s: s._use_iqrm)
    iqrm_cfg = property(lambda s: s._iqrm_cfg)

    def params(self) -> RfiParams:
        return RfiParams(self._use_mask, self._use_zero_dm, self._use_iqrm, self._iqrm_cfg.params())


class Header:
    """include/data.h:24-50 and its binding (pyapi.cpp:268-281); float fields are float."""

    def __init__(self, *args):
        if len(args) == 0:
            self._v = dict(mjd=0.0, tsamp=0.0, fch1=0.0, foff=0.0, nbits=0, nchans=0, ndata=0,
                           filename="")
        elif len(args) == 8:
            mjd, tsamp, fch1, foff, nbits, nchans, ndata, filename = args
            self._v = dict(mjd=_f32(mjd), tsamp=_f32(tsamp), fch1=_f32(fch1), foff=_f32(foff),
                           nbits=int(nbits), nchans=int(nchans), ndata=int(ndata),
                           filename=str(filename))
        elif len(args) == 1:
            o = args[0]
            self._v = dict(filename=str(o.filename), mjd=_f32(o.mjd), tsamp=_f32(o.tsamp),
                           fch1=_f32(o.fch1), foff=_f32(o.foff), nbits=int(o.nbits),
                           nchans=int(o.nchans), ndata=int(o.ndata))
        else:
            raise TypeError("Header(): expected (), 8 fields or (object)")

    mjd = property(lambda s: s._v["mjd"])
    tsamp = property(lambda s: s._v["tsamp"])
    fch1 = property(lambda s: s._v["fch1"])
    foff = property(lambda s: s._v["foff"])
    nbits = property(lambda s: s._v["nbits"])
    nchans = property(lambda s: s._v["nchans"])
    ndata = property(lambda s: s._v["ndata"])
    filename = property(lambda s: s._v["filename"])


# ------------------------------------------------------------------ result types
class DedispersedDataUint8:
    """include/data.h:52-65 and its binding (pyapi.cpp:53-95)."""

    def __init__(self):
        self._dm_times: List[np.ndarray] = []
        self._meta = dict(shape=[], dm_ndata=0, downtsample_ndata=0, dm_low=0.0, dm_high=0.0,
                          dm_step=0.0, tsample=0.0, filname="")

    dm_times = property(lambda s: list(s._dm_times))
    shape = property(lambda s: list(s._meta["shape"]))
    dm_ndata = property(lambda s: s._meta["dm_ndata"])
    downtsample_ndata = property(lambda s: s._meta["downtsample_ndata"])
    dm_low = property(lambda s: s._meta["dm_low"])
    dm_high = property(lambda s: s._meta["dm_high"])
    dm_step = property(lambda s: s._meta["dm_step"])
    tsample = property(lambda s: s._meta["tsample"])
    filname = property(lambda s: s._meta["filname"])


class DedisperedData(DedispersedDataUint8):
    """The uint64 container bound as DedisperedData (pyapi.cpp:97-130)."""


class _Spectrum:
    """Spectrum<T> (include/data.h:86-96) as bound (pyapi.cpp:135-170)."""

    def __init__(self):
        self.data = None
        self.ntimes = self.nchans = self.nbits = 0
        self.tstart = self.tend = self.dm = self.freq_start = self.freq_end = 0.0


class Spectrum8(_Spectrum):
    pass


class Spectrum16(_Spectrum):
    pass


class Spectrum32(_Spectrum):
    pass


def _fma_table(fch1: float, foff: float, n: int) -> np.ndarray:
    """fch1 + i*foff for i < n in double with one rounding (C fma), as the
    reference's reader computes it once its build (-Ofast with FMA) contracts the
    expression (src/data/filterbank.cpp:445-449)."""
    import ctypes
    import ctypes.util

    libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
    libm.fma.restype = ctypes.c_double
    libm.fma.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
    return np.array([libm.fma(float(i), float(foff), float(fch1)) for i in range(n)], np.float64)


# ------------------------------------------------------------------ SIGPROC reader
class Filterbank:
    """SIGPROC filterbank reader with the reference's behaviour
    (src/data/filterbank.cpp:64-116, 319-473): header keywords, the whole data block
    read as uint8/16/32 by nbits, and for foff < 0 the channel order reversed with
    fch1 set to the lowest frequency and foff made positive (:793-842)."""

    _INT = {"telescope_id", "machine_id", "data_type", "barycentric", "pulsarcentric",
            "nbits", "nchans", "nifs", "nbins", "ibeam", "nbeams", "npuls", "nsamples"}
    _DBL = {"az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "period", "fch1",
            "foff", "refdm"}

    def __init__(self, filename: Optional[str] = None):
        self.filename = "" if filename is None else str(filename)
        self.nchans = self.nifs = self.nbits = 0
        self.fch1 = self.foff = self.tstart = self.tsamp = 0.0
        self.ndata = 0
        self.header_size = 0
        self.use_frequence_table = False
        self.frequency_table = np.zeros(0, np.float64)
        self._data = None
        if filename is not None:
            self._read()

    def _read(self):
        with open(self.filename, "rb") as fh:
            buf = fh.read()
        pos = 0

        def get_string():
            nonlocal pos
            (n,) = struct.unpack_from("<i", buf, pos)
            s = buf[pos + 4:pos + 4 + n].decode("latin-1")
            pos += 4 + n
            return s

        if get_string() != "HEADER_START":
            raise RuntimeError("Non-Standard file format.")
        table: List[float] = []
        while True:
            key = get_string()
            if key == "HEADER_END":
                break
            if key in ("rawdatafile", "source_name"):
                get_string()
            elif key == "FREQUENCY_START":
                self.use_frequence_table = True
                table = []
            elif key == "FREQUENCY_END":
                self.nchans = len(table)
            elif key == "fchannel":
                (f,) = struct.unpack_from("<d", buf, pos)
                pos += 8
                table.append(f)
                self.use_frequence_table = True
            elif key in self._DBL:
                (v,) = struct.unpack_from("<d", buf, pos)
                pos += 8
                setattr(self, key, v)
            elif key in self._INT:
                (v,) = struct.unpack_from("<i", buf, pos)
                pos += 4
                setattr(self, key, v)
            else:
                raise RuntimeError(f"read_header - unknown parameter : {key}")
        self.header_size = pos
        if self.nifs == 0:
            self.nifs = 1
        if self.use_frequence_table and table:
            self.fch1 = self.foff = 0.0
            self.frequency_table = np.asarray(table, np.float64)
        else:
            self.frequency_table = _fma_table(self.fch1, self.foff, self.nchans)
        dt = {8: np.uint8, 16: np.uint16, 32: np.uint32}.get(self.nbits)
        if dt is None:
            raise RuntimeError(f"Unsupported nbits value: {self.nbits}")
        per = self.nifs * self.nchans
        raw = np.fromfile(self.filename, dtype=dt, offset=self.header_size)
        self.ndata = raw.size // per
        data = raw[: self.ndata * per].reshape(self.ndata, self.nifs, self.nchans)
        if self.foff < 0:
            if self.nifs != 1:
                raise RuntimeError("Only supports nifs == 1 in reverse_channanl_data")
            self.frequency_table = self.frequency_table[::-1].copy()
            if not self.use_frequence_table:
                self.fch1 = float(self.frequency_table[0])
                self.foff = abs(self.foff)
            data = data[:, :, ::-1]
        self._data = np.ascontiguousarray(data)

    @property
    def data(self) -> np.ndarray:
        return self._data

    def info(self) -> None:
        for k in ("filename", "tstart", "tsamp", "nbits", "ndata", "nifs", "nchans", "fch1", "foff"):
            print(f"{k:20s}{getattr(self, k)}")


# ------------------------------------------------------------------ helpers
def load_mask_file(path: str) -> List[int]:
    """Bad channels of a mask file as RfiMarker::load_mask reads them
    (src/rfi/rfimarker.cu:441-467): integers separated by white space, each line
    read until its first token that does not start with an integer; a missing or
    empty file means no bad channels."""
    chans: List[int] = []
    try:
        with open(path) as fh:
            lines = fh.read().splitlines()
    except OSError:
        return chans
    num = re.compile(r"^[+-]?\d+")
    for line in lines:
        for tok in line.split():
            m = num.match(tok)
            if not m or not -2 ** 31 <= int(m.group(0)) < 2 ** 31:
                break
            chans.append(int(m.group(0)))
            if m.end() != len(tok):
                break
    return chans


_PLANS: "OrderedDict[tuple, Tuple[Plan, threading.Lock]]" = OrderedDict()
_PLANS_LOCK = threading.Lock()
_MAX_PLANS = 4


@contextmanager
def _cached_plan(key, make):
    """The cached plan for `key` (made on first use), held for the caller alone.
    A plan's device workspace serves one call at a time and the library's calls
    release the GIL, so concurrent calls of one geometry take turns; the caller's
    work must be complete on the device when it leaves the block.  Plans beyond
    the newest _MAX_PLANS are closed once no call holds them."""
    while True:
        evicted = []
        with _PLANS_LOCK:
            entry = _PLANS.get(key)
            if entry is None:
                entry = (make(), threading.Lock())
                _PLANS[key] = entry
                while len(_PLANS) > _MAX_PLANS:
                    evicted.append(_PLANS.popitem(last=False)[1])
            else:
                _PLANS.move_to_end(key)
        for old_plan, old_lock in evicted:
            with old_lock:  # waits for a call that still uses it
                old_plan.close()
        plan, lock = entry
        with lock:
            if plan.closed:  # evicted between the lookup and the lock: look again
                continue
            yield plan
            return


def _as_spec_array(data) -> np.ndarray:
    """The array the reference's overloads would receive: a C-contiguous uint8,
    uint16 or uint32 array binds to its own overload unchanged; anything else
    (another dtype, a non-contiguous view, a list) reaches the first overload,
    uint8, through a forced cast (pybind11's second, converting pass)."""
    a = np.asarray(data)
    if not (a.dtype in (np.uint8, np.uint16, np.uint32) and a.flags.c_contiguous):
        a = np.ascontiguousarray(a.astype(np.uint8, casting="unsafe"))
    if a.ndim not in (1, 2, 3):
        raise RuntimeError("data must be 1D, 2D, or 3D")
    return a


def _to_device(a: np.ndarray, device: int):
    """A C-contiguous host array as a flat device tensor of the same samples; large
    arrays are copied through the library's pinned staging (dd_ingest_host: about
    four times the rate of a copy from pageable memory)."""
    if a.nbytes < (64 << 20):  # small arrays: one plain copy beats setting up the staging
        import torch

        view = {np.uint8: a, np.uint16: a.view(np.int16), np.uint32: a.view(np.int32)}[a.dtype.type]
        t = torch.from_numpy(np.ascontiguousarray(view).reshape(-1)).to(f"cuda:{device}")
        return t.view({np.uint8: torch.uint8, np.uint16: torch.uint16,
                       np.uint32: torch.uint32}[a.dtype.type])
    rows = a.reshape(-1, a.shape[-1] if a.ndim > 1 and a.shape[-1] > 0 else 1)
    return ingest.to_device(rows, device=device).view(-1)


def _result(images, dm_low, dm_high, dm_step, tsample, filname) -> DedispersedDataUint8:
    r = DedispersedDataUint8()
    r._dm_times = list(images)
    r._meta.update(shape=[512, 512, 3], dm_ndata=512, downtsample_ndata=512, dm_low=_f32(dm_low),
                   dm_high=_f32(dm_high), dm_step=_f32(dm_step), tsample=_f32(tsample),
                   filname=filname)
    return r


# ------------------------------------------------------------------ the path
def _dedisperse_spec(data, header, dm_low, dm_high, freq_start, dm_step=1, ref_freq=REF_FREQ_END,
                     time_downsample=2, t_sample=0.5, target_id=0, mask_file="mask.txt",
                     rficfg=None):
    """gpucal::dedisperse_spec<T> (src/core/dedispered.cu:988-1304) on a spectrum
    already in memory.  Positional arguments, in the order the reference's caller
    passes them: data, header, dm_low, dm_high, freq_start, freq_end, dm_step,
    time_downsample, t_sample, target_id, mask_file, rficfg."""
    # positional meaning of the bound parameters (see the module docstring)
    freq_end, dm_step_, ds = dm_step, ref_freq, time_downsample
    rfi = rficfg if rficfg is not None else RFIconfig()
    if not isinstance(header, Header):
        header = Header(header)
    a = _as_spec_array(data)
    nbits = a.dtype.itemsize * 8
    nchans, ndata = header.nchans, header.ndata
    if a.size < nchans * ndata:
        raise ValueError(f"data holds {a.size} samples, the header describes {ndata} x {nchans}")
    bad = load_mask_file(mask_file)
    hdr = dict(tsamp=header.tsamp, fch1=header.fch1, foff=header.foff, nbits=nbits,
               nchans=nchans, ndata=ndata)
    key = ("spec", nbits, nchans, ndata, header.tsamp, header.fch1, header.foff, _f32(dm_low),
           _f32(dm_high), _f32(freq_start), _f32(freq_end), _f32(dm_step_), int(ds),
           int(target_id), tuple(bad), rfi.use_mask, rfi.use_zero_dm, rfi.use_iqrm,
           tuple(vars(rfi.iqrm_cfg.params()).values()), SUBBAND_WIDTH, ZERO_DM_MODE)
    with _cached_plan(key, lambda: Plan(
            hdr, dm_low, dm_high, freq_start, freq_end, dm_step_, int(ds), algorithm="subband",
            subband_width=SUBBAND_WIDTH, ndm0=NDM0, zero_dm_mode=ZERO_DM_MODE,
            freq_mode="header", rfi=rfi.params(), bad_channels=bad,
            device=int(target_id))) as plan:
        out = plan.run(_to_device(a, int(target_id)))
        tsamp_out = _f32(header.tsamp * np.float32(ds)) if ds > 1 else header.tsamp
        # the images' copy to the host waits for the plan's work on this stream
        imgs = postprocess.device_slice_images(out, tsamp_out, 1, t_sample)
    return _result(imgs, dm_low, dm_high, dm_step_, t_sample, header.filename)


def _dedispered_fil(filename, dm_low, dm_high, freq_start, freq_end, dm_step, time_downsample,
                    t_sample, target=GPU_TARGET, target_id=0, maskfile="mask.txt", rficfg=None):
    """dedispered_fil (src/bindpy/pyapi.cpp:6-51): target 1 runs the GPU subband path
    of dedispered_fil_cuda (src/core/dedispered.cu:483-986), target 0 the CPU path
    cpucal::dedispered_fil_omp (include/cpucal.hpp:75-201), here as the brute-force
    kernel with the CPU path's semantics."""
    rfi = rficfg if rficfg is not None else RFIconfig()
    try:
        fh, table = ingest.fil_header(filename)
    except ValueError as e:  # the reference's reader raises these as RuntimeError
        raise RuntimeError(str(e)) from None
    if target not in (CPU_TARGET, GPU_TARGET):
        # the reference's switch falls through to its default for any other target
        raise RuntimeError(f"Unsupported nbits value: {fh['nbits']}")
    if fh["nifs"] == 1:
        # straight from the file into device memory (pinned staging, flip on the GPU)
        x = ingest.read_filterbank(filename, device=int(target_id))[0].view(-1)
    else:
        fil = Filterbank(filename)
        x = _to_device(fil.data.reshape(fil.ndata, -1), int(target_id))
    ndata, tsamp = fh["ndata"], fh["tsamp"]
    hdr = dict(tsamp=tsamp, fch1=fh["fch1"], foff=fh["foff"], nbits=fh["nbits"],
               nchans=fh["nchans"], ndata=ndata)
    bad = load_mask_file(maskfile)
    if target == GPU_TARGET:
        plan = Plan(hdr, dm_low, dm_high, freq_start, freq_end, dm_step, int(time_downsample),
                    algorithm="subband", subband_width=SUBBAND_WIDTH, ndm0=NDM0,
                    zero_dm_mode=ZERO_DM_MODE, freq_mode="fil", freq_table=table,
                    rfi=rfi.params(), bad_channels=bad, device=int(target_id))
        out = plan.run(x)
        ds = int(time_downsample)
        tsamp_out = _f32(tsamp * ds) if ds > 1 else _f32(tsamp)
        imgs = postprocess.device_slice_images(out, tsamp_out, 1, t_sample)
        del out
        plan.close()
        return _result(imgs, dm_low, dm_high, dm_step, t_sample, str(filename))
    plan = Plan(hdr, dm_low, dm_high, freq_start, freq_end, dm_step, int(time_downsample), t_sample,
                algorithm="brute", freq_mode="fil", freq_table=table, device=int(target_id))
    out = plan.run(x)
    # slices of std::round(t_sample / tsamp) samples, each ceil(len / ds) columns,
    # concatenated along time (include/cpucal.hpp:141-160).  The last, shorter slice
    # gets its own width; the reference reads it with the first slice's width.
    sps = int(np.floor(float(np.float32(t_sample)) / tsamp + 0.5))
    ds = int(time_downsample)
    starts, counts, off = [], [], 0
    for start in range(0, ndata, sps):
        cols = (min(start + sps, ndata) - start + ds - 1) // ds
        starts.append(off)
        counts.append(cols)
        off += cols
    imgs = postprocess.to_host_images(postprocess.device_images(out, starts, counts))
    del out
    plan.close()
    return _result(imgs, dm_low, dm_high, dm_step, t_sample, str(filename))


_SPECTRA = {8: Spectrum8, 16: Spectrum16, 32: Spectrum32}


def _single_dm(a: np.ndarray, hdr: dict, freq_mode: str, freq_table, tstart, tend, dm, freq_start,
               freq_end, maskfile, rfi: RFIconfig, nbits_out: int) -> _Spectrum:
    """One dd_single_dm_run on the flat array `a` ([ndata][nchans] samples), the
    RFI-processed rows written back into `a` as the reference's in-place masking
    leaves them."""
    from .dedisp import single_dm_spectrum

    bad = load_mask_file(maskfile)   # RfiMarkerCPU<T> reads it whether or not it is used
    nchans, ndata = int(hdr["nchans"]), int(hdr["ndata"])
    if a.size < nchans * ndata:
        raise ValueError(f"data holds {a.size} samples, the header describes {ndata} x {nchans}")
    modifies = rfi.use_iqrm or (rfi.use_mask and bool(bad))
    x = _to_device(a, 0)
    spec, g, rows = single_dm_spectrum(x, hdr, _f32(tstart), _f32(tend), _f32(dm), _f32(freq_start),
                                       _f32(freq_end), freq_mode=freq_mode, freq_table=freq_table,
                                       rfi=rfi.params(), bad_channels=bad, masked_rows=modifies)
    out = _Spectrum.__new__(_SPECTRA[a.dtype.itemsize * 8])
    _Spectrum.__init__(out)
    out.data = _to_host_same(spec)
    if modifies:
        flat = a.reshape(-1)[: ndata * nchans].reshape(ndata, nchans)
        flat[g["rfi_t0"]:g["rfi_t0"] + g["rfi_len"]] = _to_host_same(rows)
    out.ntimes, out.nchans, out.nbits = int(g["ntimes"]), int(g["nchans"]), int(nbits_out)
    out.tstart, out.tend, out.dm = _f32(tstart), _f32(g["tend"]), _f32(dm)
    out.freq_start, out.freq_end = _f32(g["freq_start"]), _f32(g["freq_end"])
    return out


def _to_host_same(t) -> np.ndarray:
    """A device tensor of uint8/16/32 samples as a numpy array of the same type."""
    import torch

    view = {torch.uint8: (torch.uint8, np.uint8), torch.uint16: (torch.int16, np.uint16),
            torch.uint32: (torch.int32, np.uint32)}[t.dtype]
    return t.view(view[0]).cpu().numpy().view(view[1])


def _dedisperse_spec_with_dm(data, header, tstart, dm, tend, freq_start, freq_end, maskfile, rficfg):
    """cpucal::dedisperse_spec_with_dm<T> (include/cpucal.hpp:341-483) through its
    binding (src/bindpy/pyapi.cpp:330-351): the spectrum of channels
    [freq_start, freq_end] over [tstart, tend) seconds, each channel shifted by its
    delay at `dm`.  The binding names its 4th and 5th parameters dm and tend while
    the C++ function takes them as tend and dm, so positionally the call is
    (data, header, tstart, tend, dm, freq_start, freq_end, maskfile, rficfg), which
    is how astroflow passes them (python/astroflow/dedispered.py:120-122).  Like the
    reference, IQRM and the mask file zero samples of `data` in place (when `data`
    is a C-contiguous uint8/16/32 array; otherwise a converted copy is masked)."""
    tstart_, tend_, dm_ = tstart, dm, tend
    if not isinstance(header, Header):
        header = Header(header)
    a = _as_spec_array(data)
    hdr = dict(tsamp=header.tsamp, fch1=header.fch1, foff=header.foff, nbits=a.dtype.itemsize * 8,
               nchans=header.nchans, ndata=header.ndata)
    return _single_dm(a, hdr, "header", None, tstart_, tend_, dm_, freq_start, freq_end, maskfile,
                      rficfg if rficfg is not None else RFIconfig(), header.nbits)


def _fil_with_dm(bits):
    def f(fil, tstart, tend, dm, freq_start, freq_end, maskfile, rficfg):
        a = fil.data if isinstance(fil, Filterbank) else None
        if a is None:
            raise RuntimeError("Filterbank holds no data")
        if a.dtype.itemsize * 8 != bits:
            # the reference reads the file's samples as the function's type whatever
            # their width, which runs past the buffer for wider types
            raise ValueError(f"the Filterbank holds {fil.nbits}-bit samples, not uint{bits}")
        hdr = dict(tsamp=fil.tsamp, fch1=fil.fch1, foff=fil.foff, nbits=bits, nchans=fil.nchans,
                   ndata=fil.ndata)
        return _single_dm(a, hdr, "fil", fil.frequency_table, tstart, tend, dm, freq_start, freq_end,
                          maskfile, rficfg if rficfg is not None else RFIconfig(), fil.nbits)
    f.__name__ = f"_dedispered_fil_with_dm_uint{bits}"
    f.__doc__ = (f"cpucal::dedispered_fil_with_dm<uint{bits}_t> (include/cpucal.hpp:203-339, "
                 "bound at src/bindpy/bindings.cpp:31-42) on a Filterbank read into memory: the "
                 "file's frequency table and double tsamp; IQRM and the mask file zero the "
                 "Filterbank's samples in place as the reference does.")
    return f


_dedispered_fil_with_dm_uint8 = _fil_with_dm(8)
_dedispered_fil_with_dm_uint16 = _fil_with_dm(16)
_dedispered_fil_with_dm_uint32 = _fil_with_dm(32)
