"""ORACLE — test infrastructure, not product code.

ctypes front end for the CPU restatement (liboracle.so, built from dd_oracle.c)
and for the reference's own code built from source (oracle/_ref/libref_cpu.so,
oracle/_ref/libref_gpu_sb<W>.so).  Only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs import this module, as the parity reference.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def reference_tree() -> str:
    """The reference source tree: $ASTROFLOW_REFERENCE, else the tree the parity
    builds in _ref were compiled from ("" when neither is known)."""
    env = os.environ.get("ASTROFLOW_REFERENCE")
    if env:
        return env
    try:
        with open(os.path.join(REF_DIR, "reference_tree.txt")) as fh:
            return fh.read().strip()
    except OSError:
        return ""

# Arithmetic variants (dd_oracle.h).  The functions' default variants are the
# forms that reproduce the reference builds; tests/test_oracle_cpu.py checks them
# against golden vectors made by those builds, and the GPU parity tests against
# the builds themselves.
FMA_DM = 1
RECIP_TSAMP = 2
RECIP_1349 = 4
FMA_VAR = 8
FMA_ZDM = 16
CPU_EXPAND = 32
CPU_EXPFMA = 64

_c_int, _c_long, _c_float, _c_double = ctypes.c_int, ctypes.c_long, ctypes.c_float, ctypes.c_double
_P = ctypes.c_void_p

_lib = None


def _np_dtype(nbits: int):
    return {8: np.uint8, 16: np.uint16, 32: np.uint32}[nbits]


def lib():
    """Load (building on demand when a compiler is present) liboracle.so."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        import subprocess

        subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
    L = ctypes.CDLL(path)
    sig = {
        "orc_freq_table_header": (None, [_c_float, _c_float, _c_int, _P]),
        "orc_freq_table_fil": (None, [_c_double, _c_double, _c_int, _P]),
        "orc_chan_range": (_c_int, [_P, _c_int, _c_float, _c_float, _P, _P]),
        "orc_dm_steps": (_c_long, [_c_float, _c_float, _c_float]),
        "orc_subband_tables_ieee": (None, [_P, _c_long, _c_long, _c_float, _c_float, _c_long,
                                           _c_int, _c_int, _c_double, _c_int, _c_int, _P, _P]),
        "orc_delay_table_fp64": (None, [_P, _c_long, _c_long, _c_float, _c_float, _c_long,
                                        _c_double, _c_int, _P]),
        "orc_cpu_delay_table": (None, [_P, _c_long, _c_long, _c_float, _c_float, _c_long,
                                       _c_double, _c_int, _P]),
        "orc_bruteforce_cpu": (_c_int, [_P, _c_int, _c_long, _c_int, _P, _c_double, _c_float,
                                        _c_float, _c_float, _c_float, _c_float, _c_int, _c_float,
                                        _c_int, _P, _P, _c_long, _P, _P, _c_long, _P]),
        "orc_subband_sums": (_c_int, [_P, _c_int, _c_long, _c_int, _c_long, _c_long, _c_int,
                                      _c_int, _c_long, _P, _P, _P]),
        "orc_time_binning": (_c_int, [_P, _c_int, _c_long, _c_int, _c_int, _P]),
        "orc_iqrm_windows": (_c_int, [_c_double, _c_double, _c_int, _c_double, ctypes.c_uint,
                                      _P, _P, _c_int]),
        "orc_iqrm_window_mask": (_c_int, [_P, _c_int, ctypes.c_uint, ctypes.c_uint,
                                          ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, _c_int,
                                          _c_float, _c_float, _c_double, _c_int, _P]),
        "orc_iqrm_lags": (_c_int, [_c_int, _c_double, _P, _c_int]),
        "orc_apply_window_masks": (None, [_P, _c_int, ctypes.c_uint, ctypes.c_uint, _c_int, _P,
                                          _P, _P]),
        "orc_zero_dm_callsite": (None, [_P, _c_int, ctypes.c_size_t, ctypes.c_size_t,
                                        ctypes.c_size_t, _c_int]),
        "orc_zero_dm_range_exact": (None, [_P, _c_int, ctypes.c_uint, ctypes.c_uint,
                                           ctypes.c_uint, ctypes.c_uint]),
        "orc_mark_channels": (None, [_P, _c_int, ctypes.c_uint, ctypes.c_uint, _P, _c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------- plan scalars
def freq_table_header(fch1: float, foff: float, nchans: int) -> np.ndarray:
    f = np.zeros(nchans, np.float64)
    lib().orc_freq_table_header(fch1, foff, nchans, _ptr(f))
    return f


def freq_table_fil(fch1: float, foff: float, nchans: int) -> np.ndarray:
    f = np.zeros(nchans, np.float64)
    lib().orc_freq_table_fil(fch1, foff, nchans, _ptr(f))
    return f


def chan_range(freq: np.ndarray, freq_start: float, freq_end: float):
    cs, ce = _c_long(), _c_long()
    rc = lib().orc_chan_range(_ptr(freq), len(freq), freq_start, freq_end, ctypes.byref(cs),
                              ctypes.byref(ce))
    if rc:
        raise ValueError("frequency range outside the band")
    return cs.value, ce.value


def dm_steps(dm_low: float, dm_high: float, dm_step: float) -> int:
    return int(lib().orc_dm_steps(dm_low, dm_high, dm_step))


@dataclass
class SubbandPlan:
    chan_start: int
    chan_end: int
    dm_steps: int
    nsamp: int
    nsb: int
    ndm_nom: int
    sb_width: int
    ndm0: int


def subband_plan(freq, nsamp_in, dm_low, dm_high, freq_start, freq_end, dm_step, ds,
                 sb_width=32, ndm0=32) -> SubbandPlan:
    cs, ce = chan_range(freq, freq_start, freq_end)
    steps = dm_steps(dm_low, dm_high, dm_step)
    dch = ce - cs + 1
    nsb = (dch + sb_width - 1) // sb_width
    return SubbandPlan(cs, ce, steps, (nsamp_in + ds - 1) // ds, nsb, (steps + ndm0 - 1) // ndm0,
                       sb_width, ndm0)


def subband_tables_ieee(freq, plan: SubbandPlan, dm_low, dm_step, tsamp, ds, variant=FMA_DM):
    dch = plan.chan_end - plan.chan_start + 1
    d1 = np.zeros((plan.ndm_nom, dch), np.int32)
    r2 = np.zeros((plan.dm_steps, plan.nsb), np.int32)
    lib().orc_subband_tables_ieee(_ptr(freq), plan.chan_start, plan.chan_end, dm_low, dm_step,
                                  plan.dm_steps, plan.sb_width, plan.ndm0, tsamp, ds, variant,
                                  _ptr(d1), _ptr(r2))
    return d1, r2


def delay_table_fp64(freq, chan_start, chan_end, dm_low, dm_step, ndm, tsamp, ds):
    d = np.zeros((ndm, chan_end - chan_start + 1), np.int32)
    lib().orc_delay_table_fp64(_ptr(freq), chan_start, chan_end, dm_low, dm_step, ndm, tsamp, ds,
                               _ptr(d))
    return d


def cpu_delay_table(freq, chan_start, chan_end, dm_low, dm_step, steps, tsamp, variant=0):
    d = np.zeros((steps, chan_end - chan_start), np.int32)
    lib().orc_cpu_delay_table(_ptr(freq), chan_start, chan_end, dm_low, dm_step, steps, tsamp,
                              variant, _ptr(d))
    return d


# ---------------------------------------------------------------- dedispersion
def bruteforce_cpu(data: np.ndarray, nchans: int, freq: np.ndarray, tsamp: float, dm_low,
                   dm_high, freq_start, freq_end, dm_step, ds, t_sample, variant=0, delay=None):
    """Raw slices of cpucal::dedispered_fil_omp; returns a list of [ndm, cols] uint64.
    `delay` ([ndm, chan_end-chan_start] int32) replaces the computed table."""
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    ndata = data.size // nchans
    steps = dm_steps(dm_low, dm_high, dm_step)
    cap = steps * (ndata + 64) + 1024
    out = np.zeros(cap, np.uint64)
    cols = np.zeros(1 << 16, np.int64)
    ns, nd = _c_long(), _c_long()
    if delay is not None:
        delay = np.ascontiguousarray(delay, np.int32)
    rc = lib().orc_bruteforce_cpu(_ptr(data), nbits, ndata, nchans, _ptr(freq), tsamp, dm_low,
                                  dm_high, freq_start, freq_end, dm_step, ds, t_sample, variant,
                                  None if delay is None else _ptr(delay), _ptr(out), cap, ctypes.byref(ns), _ptr(cols), cols.size,
                                  ctypes.byref(nd))
    if rc:
        raise ValueError(f"oracle brute force rejected the arguments (code {rc})")
    res, off = [], 0
    for s in range(ns.value):
        c = int(cols[s])
        res.append(out[off:off + nd.value * c].reshape(nd.value, c).copy())
        off += nd.value * c
    return res


def subband_sums(data: np.ndarray, nchans: int, plan: SubbandPlan, delay1, residual2):
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    nsamp = data.size // nchans
    out = np.zeros((plan.dm_steps, nsamp), np.uint64)
    d1 = np.ascontiguousarray(delay1, np.int32)
    r2 = np.ascontiguousarray(residual2, np.int32)
    rc = lib().orc_subband_sums(_ptr(data), nbits, nsamp, nchans, plan.chan_start, plan.chan_end,
                                plan.sb_width, plan.ndm0, plan.dm_steps, _ptr(d1), _ptr(r2),
                                _ptr(out))
    if rc:
        raise RuntimeError("oracle subband sums failed")
    return out


def time_binning(data: np.ndarray, nchans: int, ds: int) -> np.ndarray:
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    ndata = data.size // nchans
    out = np.zeros(((ndata + ds - 1) // ds) * nchans, data.dtype)
    lib().orc_time_binning(_ptr(data), nbits, ndata, nchans, ds, _ptr(out))
    return out.reshape(-1, nchans)


# ---------------------------------------------------------------- RFI stages
def iqrm_windows(win_sec, hop_sec, include_tail, tsamp, nsample):
    t0 = np.zeros(1 << 16, np.uint32)
    t1 = np.zeros(1 << 16, np.uint32)
    n = lib().orc_iqrm_windows(win_sec, hop_sec, int(include_tail), tsamp, nsample, _ptr(t0),
                               _ptr(t1), t0.size)
    return t0[:n].copy(), t1[:n].copy()


def iqrm_lags(radius, geofactor):
    buf = np.zeros(256, np.int32)
    n = lib().orc_iqrm_lags(radius, geofactor, _ptr(buf), 256)
    return buf[:n].copy()


def iqrm_window_mask(data, nchans, t0, t1, chan_start, chan_end, mode, radius_frac, nsigma,
                     geofactor, variant=FMA_VAR | RECIP_1349):
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    m = np.zeros(nchans, np.uint8)
    rc = lib().orc_iqrm_window_mask(_ptr(data), nbits, nchans, t0, t1, chan_start, chan_end, mode,
                                    radius_frac, nsigma, geofactor, variant, _ptr(m))
    if rc:
        raise RuntimeError(f"oracle IQRM failed ({rc})")
    return m


def iqrm_masks(data, nchans, chan_start, chan_end, tsamp, iq, variant=FMA_VAR | RECIP_1349):
    """All window masks of iqrm_cuda::rfi_iqrm_gpu; iq has mode, radius_frac, nsigma,
    geofactor, win_sec, hop_sec, include_tail.  chan_end is exclusive here."""
    nsample = np.asarray(data).size // nchans
    t0, t1 = iqrm_windows(iq.win_sec, iq.hop_sec, iq.include_tail, tsamp, nsample)
    masks = np.zeros((len(t0), nchans), np.uint8)
    for w in range(len(t0)):
        masks[w] = iqrm_window_mask(data, nchans, int(t0[w]), int(t1[w]), chan_start, chan_end,
                                    iq.mode, iq.radius_frac, iq.nsigma, iq.geofactor, variant)
    return t0, t1, masks


def apply_window_masks(data: np.ndarray, nchans, t0, t1, masks):
    nbits = data.dtype.itemsize * 8
    nsamp = data.size // nchans
    t0 = np.ascontiguousarray(t0, np.uint32)
    t1 = np.ascontiguousarray(t1, np.uint32)
    masks = np.ascontiguousarray(masks, np.uint8)
    lib().orc_apply_window_masks(_ptr(data), nbits, nchans, nsamp, len(t0), _ptr(t0), _ptr(t1),
                                 _ptr(masks))


def zero_dm_callsite(data: np.ndarray, chan_start, chan_end, down_ndata, variant=FMA_ZDM):
    lib().orc_zero_dm_callsite(_ptr(data), data.dtype.itemsize * 8, chan_start, chan_end,
                               down_ndata, variant)


def zero_dm_range_exact(data: np.ndarray, nchans, chan_start, chan_end):
    lib().orc_zero_dm_range_exact(_ptr(data), data.dtype.itemsize * 8, nchans,
                                  data.size // nchans, chan_start, chan_end)


def mark_channels(data: np.ndarray, nchans, bad):
    bad = np.ascontiguousarray(bad, np.int32)
    lib().orc_mark_channels(_ptr(data), data.dtype.itemsize * 8, nchans, data.size // nchans,
                            _ptr(bad), len(bad))


# ---------------------------------------------------------------- single-DM spectrum
@dataclass
class SingleDmGeometry:
    t_start: int
    ntimes: int
    chan_start: int
    nchans: int
    rfi_t0: int
    rfi_len: int
    tend: float
    freq_start: float
    freq_end: float
    delay: np.ndarray          # per selected channel, samples


def _lround(x: float) -> int:
    """C lround: nearest integer, halves away from zero."""
    a = abs(float(x))
    r = np.floor(a)
    r = r + 1.0 if a - r >= 0.5 else r
    return int(r if x >= 0 else -r)


def _fma_f32(a, b, c) -> np.float32:
    """fmaf(a, b, c): a*b + c rounded once to float (the reference build's -ffast-math
    contracts a*b + c into an FMA)."""
    from fractions import Fraction
    v = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
    f = np.float32(float(v))
    best = None
    for cand in (np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))):
        err = abs(Fraction(float(cand)) - v)
        key = (err, int(np.array(cand).view(np.uint32)) & 1)   # ties to even
        if best is None or key < best[0]:
            best = (key, cand)
    return np.float32(best[1])


def _fma_f64(a, b, c) -> float:
    """fma(a, b, c) in double, rounded once."""
    from fractions import Fraction
    return float(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


def single_dm_geometry(nchans, ndata, tsamp, fch1, foff, tstart, tend, dm, freq_start, freq_end,
                       fil=False, freq_table=None) -> SingleDmGeometry:
    """Window, channel selection and delays of cpucal::dedisperse_spec_with_dm
    (include/cpucal.hpp:341-427; fil=False: float tsamp/fch1/foff of a Header) and
    cpucal::dedispered_fil_with_dm (cpucal.hpp:203-286; fil=True: the file's double
    frequency table and double tsamp), in IEEE arithmetic with the two products
    followed by a sum that the reference build (-ffast-math -mfma) contracts into
    FMAs: the Header frequency table fch1 + i*foff (cpucal.hpp:374-376) and
    tend = tstart + t_len*tsamp (cpucal.hpp:459, 306).  Raises ValueError with the
    reference's message where the reference throws."""
    F = np.float32
    tstart, tend, dm, fs, fe = F(tstart), F(tend), F(dm), F(freq_start), F(freq_end)
    if not tend > tstart:
        raise ValueError("tend must be > tstart")
    if fil:
        tbl = (np.asarray(freq_table, np.float64) if freq_table is not None
               else np.array([_fma_f64(i, foff, fch1) for i in range(nchans)], np.float64))
        freq = tbl.astype(np.float32)
        t0, t1 = int(float(tstart) / tsamp), int(float(tend) / tsamp)
    else:
        tsamp = F(tsamp)
        freq = np.array([_fma_f32(F(i), F(foff), F(fch1)) for i in range(nchans)], np.float32)
        t0, t1 = int(tstart / tsamp), int(tend / tsamp)
    t_len_req = t1 - t0 if t1 > t0 else 0
    if t_len_req == 0 or t0 >= ndata:
        raise ValueError("Invalid time window for this file.")
    if not fil:
        if fs >= fe:
            raise ValueError("freq_end must be > freq_start")
        if dm < 0:
            raise ValueError("dm must be >= 0")
        if F(foff) < 0:
            raise ValueError("frequency channels are in descending order, which is not supported yet.")
    f0, fN = freq[0], freq[-1]
    fmin, fmax = min(f0, fN), max(f0, fN)
    if fs < fmin or fe > fmax or fe <= fs:
        raise ValueError("Frequency range out of file range")

    def index(f):
        raw = float(F(f - f0)) / float(F(fN - f0)) * float(nchans - 1)
        raw = min(max(raw, 0.0), float(nchans - 1))
        return int(np.floor(raw + 1e-9))

    cs, ce_incl = index(fs), index(fe)
    if ce_incl < cs:
        cs, ce_incl = ce_incl, cs
    ce = min(ce_incl + 1, nchans)
    nsel = ce - cs if ce > cs else 0
    if nsel == 0:
        raise ValueError("Empty channel selection.")
    f_high = max(freq[cs], freq[ce - 1])
    delay = np.zeros(nsel, np.int64)
    for c in range(cs, ce):
        d = F(F(F(4148.808) * dm) * F(F(1) / F(freq[c] * freq[c]) - F(1) / F(f_high * f_high)))
        delay[c - cs] = _lround(float(d) / tsamp) if fil else _lround(F(d / tsamp))
    if delay.min() < 0:
        raise ValueError("dm must be >= 0")
    dmax = int(delay.max())
    cap = ndata - t0 if ndata > t0 else 0
    t_len = min(t_len_req, cap - dmax) if cap > dmax else 0
    if t_len == 0:
        raise ValueError("Time window too short for this DM and band.")
    rfi_t0 = t0 - dmax if t0 > dmax else 0
    rfi_len = min(t_len + (t0 - rfi_t0) + 2 * dmax, ndata - rfi_t0)
    if fil:
        t_end = float(F(_fma_f64(F(t_len), tsamp, tstart)))
    else:
        t_end = float(_fma_f32(F(t_len), tsamp, tstart))
    return SingleDmGeometry(t0, t_len, cs, nsel, rfi_t0, rfi_len, t_end,
                            float(min(freq[cs], freq[ce - 1])), float(max(freq[cs], freq[ce - 1])),
                            delay)


def single_dm_spectrum(data: np.ndarray, nchans: int, g: SingleDmGeometry) -> np.ndarray:
    """The gather of cpucal.hpp:318-336 / 462-480: out[t][c] =
    data[t_start + t + delay[c]][chan_start + c]."""
    x = data.reshape(-1)[: (data.size // nchans) * nchans].reshape(-1, nchans)
    rows = g.t_start + np.arange(g.ntimes)[:, None] + g.delay[None, :]
    cols = g.chan_start + np.arange(g.nchans)[None, :]
    return x[rows, cols]


def single_dm_with_rfi(data: np.ndarray, nchans: int, g: SingleDmGeometry, tsamp: float,
                       use_mask=False, bad=(), iq=None):
    """The whole call on a copy of `data`: IQRM window masks over the RFI slice
    [rfi_t0, rfi_t0 + rfi_len) for the selected channels (cpucal.hpp:440-448,
    tsamp as the call passes it), then the mask file's channels zeroed on the same
    slice (:449-451), then the gather.  Returns (spectrum, the array after the call)."""
    x = np.ascontiguousarray(data).copy()
    flat = x.reshape(-1)[: (x.size // nchans) * nchans].reshape(-1, nchans)
    sl = flat[g.rfi_t0:g.rfi_t0 + g.rfi_len].copy()
    if iq is not None:
        t0, t1, masks = iqrm_masks(sl, nchans, g.chan_start, g.chan_start + g.nchans, tsamp, iq)
        apply_window_masks(sl, nchans, t0, t1, masks)
    if use_mask and len(bad):
        mark_channels(sl, nchans, list(bad))
    flat[g.rfi_t0:g.rfi_t0 + g.rfi_len] = sl
    return single_dm_spectrum(x, nchans, g), x


# ---------------------------------------------------------------- image step
# The reference makes its detector images with OpenCV (include/data.h:620-727):
# float slice -> cv::resize to 512x512 (INTER_AREA when both dimensions exceed the
# target, else INTER_LANCZOS4) -> cv::normalize MINMAX to uint8 -> viridis.  These
# numpy restatements fix the float arithmetic the GPU kernels (dd_images) follow;
# tests/test_image_oracle_cpu.py checks them against cv2 bit for bit.
def _area_cells(ssize: int, dsize: int):
    """Per output index: [(source index, weight)] of the area resize (overlap of the
    output cell with each source pixel over the cell width; overlaps under 1e-3
    of a pixel dropped; the last cell clipped to the source)."""
    import math
    scale = ssize / dsize
    cells = []
    for d in range(dsize):
        f1 = d * scale
        f2 = f1 + scale
        cw = min(scale, ssize - f1)
        s1 = min(math.ceil(f1), ssize - 1)
        s2 = min(math.floor(f2), ssize - 1)
        e = []
        if s1 - f1 > 1e-3:
            e.append((s1 - 1, np.float32((s1 - f1) / cw)))
        for x in range(s1, s2):
            e.append((x, np.float32(1.0 / cw)))
        if f2 - s2 > 1e-3:
            e.append((s2, np.float32(min(min(f2 - s2, 1.0), cw) / cw)))
        cells.append(e)
    return cells


def resize_area(src: np.ndarray, dh: int = 512, dw: int = 512) -> np.ndarray:
    """General-scale area resize of float32 `src`: horizontal sums in increasing
    source column, then vertical sums in increasing source row, every product and
    sum rounded to float."""
    src = np.asarray(src, np.float32)
    R, C = src.shape
    h = np.zeros((R, dw), np.float32)
    for dx, cell in enumerate(_area_cells(C, dw)):
        acc = np.zeros(R, np.float32)
        for x, w in cell:
            acc = (acc + src[:, x] * w).astype(np.float32)
        h[:, dx] = acc
    out = np.zeros((dh, dw), np.float32)
    for dy, cell in enumerate(_area_cells(R, dh)):
        acc = np.zeros(dw, np.float32)
        for y, w in cell:
            acc = (acc + h[y] * w).astype(np.float32)
        out[dy] = acc
    return out


def _lanczos4_taps(ssize: int, dsize: int):
    """Per output index: 8 clamped source indices and float weights of the
    Lanczos-4 resize (weights in double through the angle-addition form of
    sin(pi x) sin(pi x / 4) / x^2, rounded to float, times the float reciprocal of
    their float sum)."""
    import math
    F = np.float32
    r = math.sqrt(0.5)
    rot = [(1, 0), (-r, -r), (0, 1), (r, -r), (-1, 0), (r, r), (0, -1), (-r, r)]
    scale = ssize / dsize
    idx = np.zeros((dsize, 8), np.int64)
    wts = np.zeros((dsize, 8), np.float32)
    for d in range(dsize):
        f = F((d + 0.5) * scale - 0.5)
        s = int(math.floor(f))
        t = float(F(f - F(s)))
        if t < np.finfo(np.float32).eps:
            w = np.zeros(8, np.float32)
            w[3] = 1
        else:
            a0 = -(t + 3) * math.pi * 0.25
            s0, c0 = math.sin(a0), math.cos(a0)
            w = np.array([(rot[i][0] * s0 + rot[i][1] * c0) / ((-(t + 3 - i) * math.pi * 0.25) ** 2)
                          for i in range(8)]).astype(np.float32)
            tot = F(0)
            for v in w:
                tot = F(tot + v)
            w = (w * F(F(1) / tot)).astype(np.float32)
        idx[d] = [min(max(s - 3 + i, 0), ssize - 1) for i in range(8)]
        wts[d] = w
    return idx, wts


def resize_lanczos4(src: np.ndarray, dh: int = 512, dw: int = 512) -> np.ndarray:
    """Lanczos-4 resize: horizontal taps summed first to last, vertical taps last
    to first, every product and sum rounded to float."""
    src = np.asarray(src, np.float32)
    R, C = src.shape
    ix, cx = _lanczos4_taps(C, dw)
    iy, cy = _lanczos4_taps(R, dh)
    h = np.zeros((R, dw), np.float32)
    for dx in range(dw):
        acc = (src[:, ix[dx, 0]] * cx[dx, 0]).astype(np.float32)
        for k in range(1, 8):
            acc = (acc + (src[:, ix[dx, k]] * cx[dx, k]).astype(np.float32)).astype(np.float32)
        h[:, dx] = acc
    out = np.zeros((dh, dw), np.float32)
    for dy in range(dh):
        acc = (h[iy[dy, 7]] * cy[dy, 7]).astype(np.float32)
        for k in range(6, -1, -1):
            acc = (acc + (h[iy[dy, k]] * cy[dy, k]).astype(np.float32)).astype(np.float32)
        out[dy] = acc
    return out


def normalize_u8(img: np.ndarray) -> np.ndarray:
    """MINMAX to [0, 255] as uint8: scale = 255 / (max - min) in double (0 for a
    flat image), shift = -min * scale, round-half-even(fma(x, (float)scale,
    (float)shift)) clamped."""
    img = np.asarray(img, np.float32)
    mn, mx = float(img.min()), float(img.max())
    d = mx - mn
    scale = 255.0 / d if d > np.finfo(np.float64).eps else 0.0
    shift = 0.0 - mn * scale
    v = (img.astype(np.float64) * float(np.float32(scale)) + float(np.float32(shift))).astype(np.float32)
    return np.clip(np.rint(v), 0, 255).astype(np.uint8)


# ---------------------------------------------------------------- reference builds
_ref_cpu = None


def ref_cpu_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_cpu.so"))


def ref_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        L = ctypes.CDLL(os.path.join(REF_DIR, "libref_cpu.so"))
        f = L.ref_cpu_dedispered_fil_omp
        f.restype = _c_int
        f.argtypes = [_c_int, _P, _c_long, _c_int, _c_double, _c_double, _c_double, _c_float,
                      _c_float, _c_float, _c_float, _c_float, _c_int, _c_float, _P, _c_long, _P,
                      _P, _c_long, _P, ctypes.c_char_p, _c_int]
        L.ref_cpu_threads.restype = _c_int
        _ref_cpu = L
    return _ref_cpu


def ref_cpu_delays(nchans, ndata, fch1, foff, tsamp, dm_low, dm_high, freq_start, freq_end,
                   dm_step):
    """Recover the reference CPU build's [ndm, chan_end-chan_start] delay table by probing
    cpucal::dedispered_fil_omp with unit impulses (a channel-c impulse at the last sample
    shows up in DM row m at column ndata-1-delay[m][c]).  Several channels are probed per
    call, separated in time by more than the largest delay."""
    freq = freq_table_fil(fch1, foff, nchans)
    cs, ce = chan_range(freq, freq_start, freq_end)
    steps = dm_steps(dm_low, dm_high, dm_step)
    nc = ce - cs
    dmax = int(4148.808 * max(dm_high, 0) * (1 / freq[cs] ** 2 - 1 / freq[ce] ** 2) / tsamp) + 3
    span = dmax + 2
    n = max(ndata, span + 2)
    per = max(1, (n - 1) // span)
    D = np.full((steps, nc), -1, np.int64)
    for c0 in range(0, nc, per):
        chans = list(range(c0, min(nc, c0 + per)))
        y = np.zeros((n, nchans), np.uint8)
        for k, c in enumerate(chans):
            y[n - 1 - k * span, cs + c] = 1
        full = np.concatenate(ref_bruteforce_cpu(y, nchans, fch1, foff, tsamp, dm_low, dm_high,
                                                 freq_start, freq_end, dm_step, 1,
                                                 n * tsamp * 0.9999), axis=1)
        for k, c in enumerate(chans):
            t_imp = n - 1 - k * span
            lo = max(0, t_imp - dmax - 1)
            seg = full[:, lo:t_imp + 1]
            nz = seg.argmax(axis=1)
            has = seg.max(axis=1) > 0
            D[has, c] = t_imp - (lo + nz[has])
    return D.astype(np.int32)


def ref_cpu_delay_table(nchans, fch1, foff, tsamp, dm_low, dm_high, freq_start, freq_end,
                        dm_step):
    """The reference CPU build's [ndm, chan_end-chan_start] delay table, read one
    channel at a time from cpucal::dedispered_fil_omp: with 32-bit samples
    x[t][c] = t + 1 in the probed channel and zero elsewhere, output column 0 of
    DM row m is x[delay[m][c]][c] = delay[m][c] + 1.  time_downsample equal to
    the probe length makes that column the only one, so a probe costs ndm x nc
    additions and a full table takes seconds even for 1000 DMs x 1000 channels.
    Entries whose delay reaches past the probe are -1."""
    freq = freq_table_fil(fch1, foff, nchans)
    cs, ce = chan_range(freq, freq_start, freq_end)
    steps = dm_steps(dm_low, dm_high, dm_step)
    nc = ce - cs
    dmax = int(4148.808 * max(dm_high, 0) * (1 / freq[cs] ** 2 - 1 / freq[ce] ** 2) / tsamp) + 8
    n = dmax + 2
    x = np.zeros((n, nchans), np.uint32)
    ramp = np.arange(1, n + 1, dtype=np.uint32)
    cap = steps * 4 + 64
    out = np.zeros(cap, np.uint64)
    cols = np.zeros(16, np.int64)
    ns, nd = _c_long(), _c_long()
    err = ctypes.create_string_buffer(512)
    t_sample = n * tsamp * (1 - 1e-6)
    D = np.empty((steps, nc), np.int64)
    L = ref_cpu()
    for c in range(nc):
        x[:, cs + c] = ramp
        rc = L.ref_cpu_dedispered_fil_omp(32, _ptr(x), n, nchans, fch1, foff, tsamp, dm_low,
                                          dm_high, freq_start, freq_end, dm_step, n, t_sample,
                                          _ptr(out), cap, ctypes.byref(ns), _ptr(cols), cols.size,
                                          ctypes.byref(nd), err, 512)
        x[:, cs + c] = 0
        if rc:
            raise ValueError(f"reference rejected the arguments: {err.value.decode()}")
        if nd.value != steps or cols[0] != 1:
            raise RuntimeError(f"probe geometry {nd.value} rows x {cols[0]} columns")
        D[:, c] = out[:steps].astype(np.int64) - 1
    return D.astype(np.int32)


def ref_bruteforce_cpu(data, nchans, fch1, foff, tsamp, dm_low, dm_high, freq_start, freq_end,
                       dm_step, ds, t_sample):
    """The reference's cpucal::dedispered_fil_omp on a Filterbank built from `data`."""
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    ndata = data.size // nchans
    steps = dm_steps(dm_low, dm_high, dm_step)
    cap = steps * (ndata + 64) + 1024
    out = np.zeros(cap, np.uint64)
    cols = np.zeros(1 << 16, np.int64)
    ns, nd = _c_long(), _c_long()
    err = ctypes.create_string_buffer(512)
    rc = ref_cpu().ref_cpu_dedispered_fil_omp(nbits, _ptr(data), ndata, nchans, fch1, foff, tsamp,
                                              dm_low, dm_high, freq_start, freq_end, dm_step, ds,
                                              t_sample, _ptr(out), cap, ctypes.byref(ns),
                                              _ptr(cols), cols.size, ctypes.byref(nd), err, 512)
    if rc:
        raise ValueError(f"reference rejected the arguments: {err.value.decode()}")
    res, off = [], 0
    for s in range(ns.value):
        c = int(cols[s])
        res.append(out[off:off + nd.value * c].reshape(nd.value, c).copy())
        off += nd.value * c
    return res


class _TapRfi(ctypes.Structure):
    _fields_ = [("use_mask", _c_int), ("use_zero_dm", _c_int), ("use_iqrm", _c_int),
                ("iq_mode", _c_int), ("iq_radius_frac", _c_float), ("iq_nsigma", _c_float),
                ("iq_geofactor", _c_double), ("iq_win_sec", _c_double), ("iq_hop_sec", _c_double),
                ("iq_include_tail", _c_int)]


def _tap_rfi(use_mask, use_zero_dm, use_iqrm, iq):
    r = _TapRfi()
    r.use_mask, r.use_zero_dm, r.use_iqrm = int(use_mask), int(use_zero_dm), int(use_iqrm)
    if iq is not None:
        r.iq_mode, r.iq_radius_frac, r.iq_nsigma = iq.mode, iq.radius_frac, iq.nsigma
        r.iq_geofactor, r.iq_win_sec, r.iq_hop_sec = iq.geofactor, iq.win_sec, iq.hop_sec
        r.iq_include_tail = int(iq.include_tail)
    else:
        r.iq_mode, r.iq_radius_frac, r.iq_nsigma, r.iq_geofactor = 0, 0.1, 3.0, 1.5
        r.iq_win_sec, r.iq_hop_sec, r.iq_include_tail = 5.0, 2.5, 1
    return r


_ref_gpu = {}


def ref_gpu_available(sb_width: int) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_gpu_sb{sb_width}.so"))


def ref_gpu(sb_width: int):
    if sb_width not in _ref_gpu:
        L = ctypes.CDLL(os.path.join(REF_DIR, f"libref_gpu_sb{sb_width}.so"))
        L.ref_gpu_dedisperse_spec.restype = _c_int
        L.ref_gpu_dedisperse_spec.argtypes = [
            _c_int, _P, _c_float, _c_float, _c_float, _c_float, _c_int, _c_long, _c_float,
            _c_float, _c_float, _c_float, _c_float, _c_int, _c_float, _c_int, ctypes.c_char_p, _P,
            _P, _c_long, _P, _P, ctypes.c_char_p, _c_int]
        L.ref_gpu_tables.restype = _c_int
        L.ref_gpu_tables.argtypes = [_c_float, _c_float, _c_float, _c_int, _c_long, _c_float,
                                     _c_float, _c_float, _c_float, _c_float, _c_int, _P, _c_long,
                                     _P, _c_long, _P, ctypes.c_char_p, _c_int]
        L.ref_gpu_rfi.restype = _c_int
        L.ref_gpu_rfi.argtypes = [_c_int, _P, _c_float, _c_float, _c_float, _c_int, _c_long,
                                  _c_float, _c_float, _c_int, ctypes.c_char_p, _P, _P, _c_long, _P,
                                  _P, _P, _c_long, _P, _P, ctypes.c_char_p, _c_int]
        L.ref_gpu_dedispered_fil.restype = _c_int
        L.ref_gpu_dedispered_fil.argtypes = [
            ctypes.c_char_p, _c_float, _c_float, _c_float, _c_float, _c_float, _c_int, _c_float,
            _c_int, ctypes.c_char_p, _P, _P, _c_long, _P, _P, ctypes.c_char_p, _c_int]
        L.ref_set_capture_sink.restype = None
        L.ref_set_capture_sink.argtypes = [_P, _P, _c_long]
        L.ref_capture_elem.restype = _c_long
        L.ref_capture_elem.argtypes = []
        L.ref_gpu_zero_dm_range.restype = _c_int
        L.ref_gpu_zero_dm_range.argtypes = [_c_int, _P, _c_int, _c_long, _c_int, _c_int, _P,
                                            ctypes.c_char_p, _c_int]
        _ref_gpu[sb_width] = L
    return _ref_gpu[sb_width]


def ref_gpu_dedisperse_spec_rows(data, nchans, tsamp, fch1, foff, dm_low, dm_high, freq_start,
                                 freq_end, dm_step, ds, rows=None, t_sample=0.5, sb_width=32,
                                 mask_file="", use_mask=False, use_zero_dm=False, use_iqrm=False,
                                 iq=None, device=0):
    """Rows of the raw [dm_steps, down_ndata] output of the reference's
    gpucal::dedisperse_spec, captured in the output's own type (uint32, or uint64
    for 32-bit samples) without the widened host copy, so chunks of 10^9 output
    samples fit in host memory.  rows: DM-row indices (None: all rows)."""
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    ndata = data.size // nchans
    steps = dm_steps(dm_low, dm_high, dm_step)
    cols = (ndata + ds - 1) // ds
    sel = np.arange(steps, dtype=np.int64) if rows is None else np.asarray(rows, dtype=np.int64)
    out = np.zeros((sel.size, cols), np.uint64 if nbits == 32 else np.uint32)
    L = ref_gpu(sb_width)
    nr, nc = _c_long(), _c_long()
    err = ctypes.create_string_buffer(512)
    r = _tap_rfi(use_mask, use_zero_dm, use_iqrm, iq)
    L.ref_set_capture_sink(_ptr(out), _ptr(sel), 0 if rows is None else int(sel.size))
    try:
        rc = L.ref_gpu_dedisperse_spec(
            nbits, _ptr(data), 0.0, tsamp, fch1, foff, nchans, ndata, dm_low, dm_high, freq_start,
            freq_end, dm_step, ds, t_sample, device, mask_file.encode(), ctypes.byref(r), None, 0,
            ctypes.byref(nr), ctypes.byref(nc), err, 512)
        elem = L.ref_capture_elem()
    finally:
        L.ref_set_capture_sink(None, None, 0)
    if rc:
        raise ValueError(f"reference GPU call failed: {err.value.decode()}")
    if (nr.value, nc.value) != (steps, cols) or elem != out.itemsize:
        raise RuntimeError(f"reference output {nr.value}x{nc.value} of {elem}-byte elements, "
                           f"expected {steps}x{cols} of {out.itemsize}")
    return out


def ref_gpu_zero_dm_range(data, nchans, chan_start, chan_end, sb_width=32):
    """The reference's range zero-DM filter (RfiMarker<T>::zero_dm_filter with a
    channel range, src/rfi/rfimarker.cu:257-305) applied to a copy of `data`."""
    data = np.ascontiguousarray(data)
    out = np.empty_like(data)
    err = ctypes.create_string_buffer(512)
    rc = ref_gpu(sb_width).ref_gpu_zero_dm_range(data.dtype.itemsize * 8, _ptr(data), nchans,
                                                 data.size // nchans, chan_start, chan_end,
                                                 _ptr(out), err, 512)
    if rc:
        raise ValueError(f"reference zero-DM failed: {err.value.decode()}")
    return out


def ref_gpu_dedisperse_spec(data, nchans, tsamp, fch1, foff, dm_low, dm_high, freq_start,
                            freq_end, dm_step, ds, t_sample=0.5, sb_width=32, mask_file="",
                            use_mask=False, use_zero_dm=False, use_iqrm=False, iq=None,
                            device=0):
    """Raw [dm_steps, down_ndata] output of the reference's gpucal::dedisperse_spec."""
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    ndata = data.size // nchans
    steps = dm_steps(dm_low, dm_high, dm_step)
    cap = steps * ((ndata + ds - 1) // ds)
    out = np.zeros(cap, np.uint64)
    rows, cols = _c_long(), _c_long()
    err = ctypes.create_string_buffer(512)
    r = _tap_rfi(use_mask, use_zero_dm, use_iqrm, iq)
    rc = ref_gpu(sb_width).ref_gpu_dedisperse_spec(
        nbits, _ptr(data), 0.0, tsamp, fch1, foff, nchans, ndata, dm_low, dm_high, freq_start,
        freq_end, dm_step, ds, t_sample, device, mask_file.encode(), ctypes.byref(r), _ptr(out),
        cap, ctypes.byref(rows), ctypes.byref(cols), err, 512)
    if rc:
        raise ValueError(f"reference GPU call failed: {err.value.decode()}")
    return out[:rows.value * cols.value].reshape(rows.value, cols.value)


def ref_gpu_timed_available(sb_width: int) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_gpu_timed_sb{sb_width}.so"))


def ref_gpu_time_spec(data, nchans, tsamp, fch1, foff, dm_low, dm_high, freq_start, freq_end,
                      dm_step, ds, t_sample=0.5, sb_width=64, use_mask=False, use_zero_dm=False,
                      use_iqrm=False, iq=None, device=0):
    """One call of the reference's gpucal::dedisperse_spec from its timing build:
    returns (rows, cols, {timer label: ms}) from the reference's own AF_DEBUG
    timers (CUDA events around H2D, binning, IQRM, zero-DM, stage 1, stage 2,
    D2H) plus "wall" (host time of the whole call)."""
    import re
    import tempfile
    import time

    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    ndata = data.size // nchans
    L = ctypes.CDLL(os.path.join(REF_DIR, f"libref_gpu_timed_sb{sb_width}.so"))
    L.ref_gpu_dedisperse_spec.restype = _c_int
    L.ref_gpu_dedisperse_spec.argtypes = [
        _c_int, _P, _c_float, _c_float, _c_float, _c_float, _c_int, _c_long, _c_float,
        _c_float, _c_float, _c_float, _c_float, _c_int, _c_float, _c_int, ctypes.c_char_p, _P,
        _P, _c_long, _P, _P, ctypes.c_char_p, _c_int]
    rows, cols = _c_long(), _c_long()
    err = ctypes.create_string_buffer(512)
    r = _tap_rfi(use_mask, use_zero_dm, use_iqrm, iq)
    libc = ctypes.CDLL(None)
    with tempfile.TemporaryFile(mode="w+b") as tf:
        libc.fflush(None)
        saved = os.dup(1)
        os.dup2(tf.fileno(), 1)
        try:
            t0 = time.perf_counter()
            rc = L.ref_gpu_dedisperse_spec(
                nbits, _ptr(data), 0.0, tsamp, fch1, foff, nchans, ndata, dm_low, dm_high,
                freq_start, freq_end, dm_step, ds, t_sample, device, b"", ctypes.byref(r), None,
                0, ctypes.byref(rows), ctypes.byref(cols), err, 512)
            wall = (time.perf_counter() - t0) * 1e3
            libc.fflush(None)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        tf.seek(0)
        text = tf.read().decode(errors="replace")
    if rc:
        raise ValueError(f"reference GPU call failed: {err.value.decode()}")
    timers = {m.group(1).strip(): float(m.group(2))
              for m in re.finditer(r"\[TIMER\]\s*(.+?)\s*:\s*([0-9.]+)\s*ms", text)}
    timers["wall"] = wall
    return rows.value, cols.value, timers


def ref_gpu_dedispered_fil(filename, dm_low, dm_high, freq_start, freq_end, dm_step, ds,
                           t_sample=0.5, sb_width=32, mask_file="", use_mask=False,
                           use_zero_dm=False, use_iqrm=False, iq=None, cap=1 << 22, device=0):
    """Raw [dm_steps, down_ndata] output of the reference's file entry point
    (Filterbank reader + gpucal::dedispered_fil_cuda)."""
    out = np.zeros(cap, np.uint64)
    rows, cols = _c_long(), _c_long()
    err = ctypes.create_string_buffer(512)
    r = _tap_rfi(use_mask, use_zero_dm, use_iqrm, iq)
    rc = ref_gpu(sb_width).ref_gpu_dedispered_fil(
        str(filename).encode(), dm_low, dm_high, freq_start, freq_end, dm_step, ds, t_sample,
        device, mask_file.encode(), ctypes.byref(r), _ptr(out), cap, ctypes.byref(rows),
        ctypes.byref(cols), err, 512)
    if rc:
        raise ValueError(f"reference GPU call failed: {err.value.decode()}")
    return out[:rows.value * cols.value].reshape(rows.value, cols.value)


def ref_gpu_spec_with_dm(data, nchans, tsamp, fch1, foff, tstart, tend, dm, freq_start, freq_end,
                         mask_file="", use_mask=False, use_iqrm=False, iq=None, sb_width=32):
    """The reference's cpucal::dedisperse_spec_with_dm on a copy of `data`; returns
    (spectrum [ntimes, nsel], (tstart, tend, freq_start, freq_end), the copy after the
    call (the reference zeroes the RFI-masked samples of its input in place))."""
    data = np.ascontiguousarray(data).copy()
    nbits = data.dtype.itemsize * 8
    L = ref_gpu(sb_width)
    L.ref_gpu_spec_with_dm.restype = _c_int
    L.ref_gpu_spec_with_dm.argtypes = [_c_int, _P, _c_float, _c_float, _c_float, _c_int, _c_long,
                                       _c_float, _c_float, _c_float, _c_float, _c_float,
                                       ctypes.c_char_p, _P, _P, _c_long, _P, _P, _P,
                                       ctypes.c_char_p, _c_int]
    r = _tap_rfi(use_mask, False, use_iqrm, iq)
    cap = data.size
    raw = np.zeros(cap, data.dtype)
    nt, ns = _c_long(), _c_long()
    meta = np.zeros(4, np.float32)
    err = ctypes.create_string_buffer(512)
    rc = L.ref_gpu_spec_with_dm(nbits, _ptr(data), tsamp, fch1, foff, nchans, data.size // nchans,
                                tstart, tend, dm, freq_start, freq_end, mask_file.encode(),
                                ctypes.byref(r), _ptr(raw), cap, ctypes.byref(nt), ctypes.byref(ns),
                                _ptr(meta), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return raw[:nt.value * ns.value].reshape(nt.value, ns.value), tuple(meta), data


def ref_gpu_fil_with_dm(filename, nbits, tstart, tend, dm, freq_start, freq_end, mask_file="",
                        use_mask=False, use_iqrm=False, iq=None, cap=1 << 26, sb_width=32):
    """The reference's Filterbank + cpucal::dedispered_fil_with_dm."""
    L = ref_gpu(sb_width)
    L.ref_gpu_fil_with_dm.restype = _c_int
    L.ref_gpu_fil_with_dm.argtypes = [ctypes.c_char_p, _c_float, _c_float, _c_float, _c_float,
                                      _c_float, ctypes.c_char_p, _P, _P, _c_long, _P, _P, _P,
                                      ctypes.c_char_p, _c_int]
    r = _tap_rfi(use_mask, False, use_iqrm, iq)
    raw = np.zeros(cap, {8: np.uint8, 16: np.uint16, 32: np.uint32}[nbits])
    nt, ns = _c_long(), _c_long()
    meta = np.zeros(4, np.float32)
    err = ctypes.create_string_buffer(512)
    rc = L.ref_gpu_fil_with_dm(str(filename).encode(), tstart, tend, dm, freq_start, freq_end,
                               mask_file.encode(), ctypes.byref(r), _ptr(raw), cap, ctypes.byref(nt),
                               ctypes.byref(ns), _ptr(meta), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return raw[:nt.value * ns.value].reshape(nt.value, ns.value), tuple(meta)


def ref_gpu_tables(nchans, ndata, tsamp, fch1, foff, dm_low, dm_high, freq_start, freq_end,
                   dm_step, ds, sb_width=32):
    steps = dm_steps(dm_low, dm_high, dm_step)
    cap1 = ((steps + 31) // 32 + 1) * nchans
    cap2 = steps * (nchans // 1 + 1)
    d1 = np.zeros(cap1, np.int32)
    r2 = np.zeros(cap2, np.int32)
    info = np.zeros(8, np.int64)
    err = ctypes.create_string_buffer(512)
    rc = ref_gpu(sb_width).ref_gpu_tables(tsamp, fch1, foff, nchans, ndata, dm_low, dm_high,
                                          freq_start, freq_end, dm_step, ds, _ptr(d1), cap1,
                                          _ptr(r2), cap2, _ptr(info), err, 512)
    if rc:
        raise ValueError(f"reference table build failed: {err.value.decode()}")
    cs, ce, st_, nout, nsb, ndm_nom = (int(v) for v in info[:6])
    dch = ce - cs + 1
    return (d1[:ndm_nom * dch].reshape(ndm_nom, dch).copy(),
            r2[:st_ * nsb].reshape(st_, nsb).copy(), dict(chan_start=cs, chan_end=ce,
                                                          dm_steps=st_, nsamp=nout, nsb=nsb,
                                                          ndm_nom=ndm_nom))


def ref_gpu_rfi(data, nchans, tsamp, fch1, foff, freq_start, freq_end, ds, mask_file="",
                use_mask=False, use_zero_dm=False, use_iqrm=False, iq=None, sb_width=32):
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    ndata = data.size // nchans
    nout = (ndata + ds - 1) // ds
    out = np.zeros(nout * nchans, data.dtype)
    wcap = 4096
    t0 = np.zeros(wcap, np.uint32)
    t1 = np.zeros(wcap, np.uint32)
    wm = np.zeros(wcap * nchans, np.uint8)
    nwin = _c_long()
    info = np.zeros(4, np.int64)
    err = ctypes.create_string_buffer(512)
    r = _tap_rfi(use_mask, use_zero_dm, use_iqrm, iq)
    rc = ref_gpu(sb_width).ref_gpu_rfi(nbits, _ptr(data), tsamp, fch1, foff, nchans, ndata,
                                       freq_start, freq_end, ds, mask_file.encode(),
                                       ctypes.byref(r), _ptr(out), out.size, _ptr(t0), _ptr(t1),
                                       _ptr(wm), wcap, ctypes.byref(nwin), _ptr(info), err, 512)
    if rc:
        raise ValueError(f"reference RFI replay failed: {err.value.decode()}")
    n = nwin.value
    return (out.reshape(nout, nchans), t0[:n].copy(), t1[:n].copy(),
            wm[:n * nchans].reshape(n, nchans).copy())
