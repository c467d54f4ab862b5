"""The drop-in module astroflow_b200._astroflow_core on the host: constructors and
attributes of the bound types (src/bindpy/pyapi.cpp:194-281, include/rfi.h,
include/data.h:24-50), the SIGPROC reader (src/data/filterbank.cpp), mask files
(src/rfi/rfimarker.cu:441-467), argument handling of _dedisperse_spec
(src/bindpy/bindings.cpp:43-57) and the slice arithmetic of the image step
(include/data.h:640-643).  Nothing here needs a GPU."""
import types

import numpy as np
import pytest

from astroflow_b200 import _astroflow_core as C
from astroflow_b200 import postprocess
from oracle import cv2_images as CVI
from sigproc_writer import write_fil

F32 = np.float32


def test_iqrmconfig_constructors():
    d = C.IQRMconfig()
    assert (d.mode, d.nsigma, d.geofactor, d.win_sec, d.hop_sec, d.include_tail) == (0, 3.0, 1.5, 5.0, 2.5, True)
    assert d.radius_frac == float(F32(0.10))
    # init<int, float x5, bool>: every real passes through float
    c = C.IQRMconfig(1, 0.1, 2.7, 1.3, 0.1, 0.05, False)
    assert c.mode == 1 and c.include_tail is False
    for got, want in ((c.radius_frac, 0.1), (c.nsigma, 2.7), (c.geofactor, 1.3), (c.win_sec, 0.1), (c.hop_sec, 0.05)):
        assert got == float(F32(want))
    # init<py::object>: radius_frac/nsigma as float, the rest as double
    o = types.SimpleNamespace(mode=0, radius_frac=0.3, nsigma=4.1, geofactor=1.7, win_sec=0.3,
                              hop_sec=0.15, include_tail=1)
    p = C.IQRMconfig(o)
    assert p.radius_frac == float(F32(0.3)) and p.nsigma == float(F32(4.1))
    assert (p.geofactor, p.win_sec, p.hop_sec, p.include_tail) == (1.7, 0.3, 0.15, True)
    with pytest.raises(TypeError):
        C.IQRMconfig(1, 2)


def test_rficonfig_constructors():
    r = C.RFIconfig()
    assert (r.use_mask, r.use_zero_dm, r.use_iqrm) == (False, False, False)
    iq = C.IQRMconfig(0, 0.2, 3.0, 1.5, 0.0, 0.0, True)
    r = C.RFIconfig(True, False, True, iq)
    assert (r.use_mask, r.use_zero_dm, r.use_iqrm) == (True, False, True)
    assert r.iqrm_cfg.radius_frac == float(F32(0.2))
    o = types.SimpleNamespace(use_mask=0, use_zero_dm=1, use_iqrm=1,
                              iqrm_cfg=types.SimpleNamespace(mode=1, radius_frac=0.05, nsigma=3.0,
                                                             geofactor=1.5, win_sec=0.0,
                                                             hop_sec=0.0, include_tail=True))
    r = C.RFIconfig(o)
    assert (r.use_mask, r.use_zero_dm, r.use_iqrm, r.iqrm_cfg.mode) == (False, True, True, 1)
    p = r.params()
    assert p.use_zero_dm and p.iqrm.mode == 1


def test_header_constructors_round_to_float():
    h = C.Header(60000.123456789, 49.152e-6, 1000.1220703125, 0.1220703125, 8, 4096, 1 << 20, "x.fil")
    assert h.mjd == float(F32(60000.123456789)) and h.tsamp == float(F32(49.152e-6))
    assert (h.nbits, h.nchans, h.ndata, h.filename) == (8, 4096, 1 << 20, "x.fil")
    h2 = C.Header(types.SimpleNamespace(mjd=1.0, tsamp=1e-4, fch1=1200.3, foff=0.7, nbits=16,
                                        nchans=64, ndata=100, filename="y"))
    assert h2.fch1 == float(F32(1200.3)) and h2.nbits == 16
    assert C.Header().nchans == 0


def test_filterbank_reader_flips_descending_band(tmp_path):
    rng = np.random.default_rng(1)
    data = rng.integers(0, 256, size=(50, 16)).astype(np.uint8)
    p = tmp_path / "desc.fil"
    write_fil(p, data, 64e-6, 1500.0, -2.0)
    fil = C.Filterbank(str(p))
    assert (fil.nchans, fil.nifs, fil.nbits, fil.ndata) == (16, 1, 8, 50)
    assert fil.fch1 == 1500.0 - 15 * 2.0 and fil.foff == 2.0
    assert np.array_equal(fil.frequency_table, 1500.0 - 2.0 * np.arange(16)[::-1])
    assert fil.data.shape == (50, 1, 16)
    assert np.array_equal(fil.data[:, 0, :], data[:, ::-1])


def test_filterbank_reader_ascending_16bit_and_table(tmp_path):
    rng = np.random.default_rng(2)
    data = rng.integers(0, 65536, size=(33, 8)).astype(np.uint16)
    p = tmp_path / "asc.fil"
    write_fil(p, data, 1e-4, 1100.0, 0.5, extra=[("refdm", 12.5), ("ibeam", 3), ("rawdatafile", "a.raw")])
    fil = C.Filterbank(str(p))
    assert (fil.nbits, fil.ndata, fil.fch1, fil.foff) == (16, 33, 1100.0, 0.5)
    assert np.array_equal(fil.data[:, 0, :], data)
    # an explicit frequency table sets fch1 = foff = 0 and is kept in file order
    table = 1000.0 + np.arange(8) * 3.0
    p2 = tmp_path / "table.fil"
    write_fil(p2, data, 1e-4, 0, 0, freq_table=table)
    fil2 = C.Filterbank(str(p2))
    assert (fil2.fch1, fil2.foff, fil2.nchans) == (0.0, 0.0, 8)
    assert np.array_equal(fil2.frequency_table, table)


def test_filterbank_reader_rejects_unknown_keyword(tmp_path):
    data = np.zeros((4, 4), np.uint8)
    p = tmp_path / "bad.fil"
    write_fil(p, data, 1e-4, 1100.0, 0.5, extra=[("not_a_key", 1)])
    with pytest.raises(RuntimeError, match="unknown parameter"):
        C.Filterbank(str(p))


def test_mask_file_parsing(tmp_path):
    p = tmp_path / "mask.txt"
    p.write_text("3 5 7\n  11\t12 x 99\n\n-1 4096 20abc 21\n")
    assert C.load_mask_file(str(p)) == [3, 5, 7, 11, 12, -1, 4096, 20]
    assert C.load_mask_file(str(tmp_path / "missing.txt")) == []


def test_spec_array_follows_overload_resolution():
    a = np.arange(12, dtype=np.uint16).reshape(3, 4)
    assert C._as_spec_array(a).dtype == np.uint16
    assert C._as_spec_array(a.astype(np.uint32)).dtype == np.uint32
    # a non-contiguous view or another dtype reaches the uint8 overload by a forced cast
    v = (np.arange(24, dtype=np.uint16) + 250).reshape(4, 6)[:, ::2]
    got = C._as_spec_array(v)
    assert got.dtype == np.uint8 and np.array_equal(got, v.astype(np.uint8))
    assert C._as_spec_array([[1.0, 2.0]]).dtype == np.uint8
    with pytest.raises(RuntimeError, match="1D, 2D, or 3D"):
        C._as_spec_array(np.zeros((1, 1, 1, 1), np.uint8))


def test_samples_per_slice_float_arithmetic():
    # (size_t)(slice_duration / (tsamp * ds)) evaluated in float
    assert postprocess.samples_per_slice(49.152e-6, 1, 0.5) == int(F32(0.5) / F32(49.152e-6))
    assert postprocess.samples_per_slice(1e-4, 4, 0.1) == int(F32(0.1) / (F32(1e-4) * F32(4)))


def test_slice_arithmetic_equals_the_oracle():
    for ts, ds, dur in [(49.152e-6, 1, 0.5), (1e-4, 4, 0.1), (64e-6, 2, 0.5), (1.26646875e-3, 3, 0.3)]:
        assert postprocess.samples_per_slice(ts, ds, dur) == CVI.samples_per_slice(ts, ds, dur)


def test_oracle_slice_images_shapes_and_colormap():
    pytest.importorskip("cv2")
    rng = np.random.default_rng(0)
    raw = rng.integers(0, 1000, size=(40, 250)).astype(np.uint32)
    imgs = CVI.slice_images(raw, 1e-3, 1, 0.1)
    assert len(imgs) == 3 and all(i.shape == (512, 512, 3) and i.dtype == np.uint8 for i in imgs)
    import cv2

    # min-max normalisation: the smallest and largest sums map to viridis(0) and viridis(255)
    ramp = CVI.images([np.arange(600 * 600, dtype=np.uint32).reshape(600, 600)])[0]
    lut = cv2.applyColorMap(np.array([[0, 255]], np.uint8), cv2.COLORMAP_VIRIDIS)[0]
    assert np.array_equal(ramp[0, 0], lut[0]) and np.array_equal(ramp[-1, -1], lut[1])


def test_dedisperse_spec_arguments_are_positional_like_the_reference():
    import inspect

    names = list(inspect.signature(C._dedisperse_spec).parameters)
    assert names == ["data", "header", "dm_low", "dm_high", "freq_start", "dm_step", "ref_freq",
                     "time_downsample", "t_sample", "target_id", "mask_file", "rficfg"]
    names = list(inspect.signature(C._dedispered_fil).parameters)
    assert names == ["filename", "dm_low", "dm_high", "freq_start", "freq_end", "dm_step",
                     "time_downsample", "t_sample", "target", "target_id", "maskfile", "rficfg"]
    # bindings.cpp:59-61 names the 4th and 5th parameters dm, tend (positionally tend, dm)
    names = list(inspect.signature(C._dedisperse_spec_with_dm).parameters)
    assert names == ["data", "header", "tstart", "dm", "tend", "freq_start", "freq_end",
                     "maskfile", "rficfg"]
    names = list(inspect.signature(C._dedispered_fil_with_dm_uint16).parameters)
    assert names == ["fil", "tstart", "tend", "dm", "freq_start", "freq_end", "maskfile", "rficfg"]


def test_dedispered_fil_unknown_target_raises_like_the_reference(tmp_path):
    p = tmp_path / "t.fil"
    write_fil(p, np.zeros((16, 4), np.uint8), 1e-4, 1100.0, 0.5)
    with pytest.raises(RuntimeError, match="Unsupported nbits value: 8"):
        C._dedispered_fil(str(p), 0, 10, 1100.0, 1101.5, 1, 1, 0.001, target=7)


def test_single_dm_fil_entry_points_check_the_sample_width(tmp_path):
    """_dedispered_fil_with_dm_uint{8,16,32} read the Filterbank's samples as their
    own type; a file of another width is refused before any device work."""
    p = tmp_path / "a.fil"
    write_fil(str(p), np.zeros((64, 8), np.uint8), 1e-3, 1000.0, 1.0)
    fb = C.Filterbank(str(p))
    for f in (C._dedispered_fil_with_dm_uint16, C._dedispered_fil_with_dm_uint32):
        with pytest.raises(ValueError):
            f(fb, 0.0, 0.01, 1.0, 1000.0, 1007.0, "", C.RFIconfig())
    with pytest.raises(RuntimeError):
        C._dedispered_fil_with_dm_uint8(None, 0.0, 0.01, 1.0, 1000.0, 1007.0, "", C.RFIconfig())


def test_viridis_table_is_the_reference_colormap():
    """The GPU image step colors through a 256-entry table; it must equal
    cvtColor(GRAY2RGB) + applyColorMap(VIRIDIS) (include/data.h:703-705)."""
    cv2 = pytest.importorskip("cv2")
    lut = postprocess.viridis_lut()
    g = np.random.default_rng(3).integers(0, 256, (64, 80), dtype=np.uint8)
    want = cv2.applyColorMap(cv2.cvtColor(g, cv2.COLOR_GRAY2RGB), cv2.COLORMAP_VIRIDIS)
    assert lut.shape == (256, 3) and np.array_equal(lut[g], want)


class _FakePlan:
    def __init__(self, log):
        self.log, self.closed = log, False

    def close(self):
        self.log.append("close")
        self.closed = True


def test_plan_cache_serialises_calls_and_closes_evicted_plans(monkeypatch):
    """Calls of one geometry hold the cached plan one at a time; plans past the
    newest _MAX_PLANS are closed, after the call that holds one has finished."""
    import threading
    import time
    from collections import OrderedDict

    monkeypatch.setattr(C, "_PLANS", OrderedDict())
    log = []
    inside, overlap = [0], [False]
    lock = threading.Lock()

    def call(key):
        with C._cached_plan(key, lambda: _FakePlan(log)) as p:
            with lock:
                inside[0] += 1
                overlap[0] |= inside[0] > 1
            time.sleep(0.02)
            with lock:
                inside[0] -= 1
            assert not p.closed

    threads = [threading.Thread(target=call, args=(("k",),)) for _ in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not overlap[0] and log == []

    # a call holding the oldest plan delays its closing until the call ends
    held = threading.Event()
    release = threading.Event()

    def holder():
        with C._cached_plan(("k",), lambda: _FakePlan(log)):
            held.set()
            release.wait(5)
            log.append("holder done")

    h = threading.Thread(target=holder)
    h.start()
    held.wait(5)
    evictor = threading.Thread(
        target=lambda: [call((f"n{i}",)) for i in range(C._MAX_PLANS)])
    evictor.start()
    time.sleep(0.1)
    assert log == []  # the eviction waits for the holder
    release.set()
    h.join()
    evictor.join()
    assert log == ["holder done", "close"]
    assert len(C._PLANS) == C._MAX_PLANS and ("k",) not in C._PLANS
