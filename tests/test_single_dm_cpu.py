"""Single-DM dedispersed spectra (cpucal::dedisperse_spec_with_dm and
cpucal::dedispered_fil_with_dm, include/cpucal.hpp:203-483) on the CPU: the
oracle against the reference's golden fixtures and, where the reference builds
exist, against the reference itself; the library's host-side geometry
(dd_single_dm_geometry) against the oracle."""
import ctypes
import glob
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from sigproc_writer import write_fil

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_single_*.npz")))
F32 = np.float32


class _Iq:
    def __init__(self, mode, radius_frac, nsigma, win_sec, hop_sec):
        self.mode, self.radius_frac, self.nsigma = int(mode), radius_frac, nsigma
        self.geofactor, self.win_sec, self.hop_sec, self.include_tail = 1.5, win_sec, hop_sec, True


def fixture_case(path):
    """The fixture's call as (data in ascending channel order, geometry args)."""
    z = np.load(path)
    x, nchans, fil = z["data"], int(z["nchans"]), bool(z["fil"])
    fch1, foff = float(z["fch1"]), float(z["foff"])
    if foff < 0:   # the reader turns a descending file around (filterbank.cpp:793-842)
        x = np.ascontiguousarray(x[:, ::-1])
        fch1, foff = fch1 + (nchans - 1) * foff, -foff
    iq = _Iq(*z["iq"]) if z["iq"].size else None
    return z, x, nchans, fil, fch1, foff, iq


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[11:-4] for p in FIXTURES])
def test_oracle_matches_golden(path):
    z, x, nchans, fil, fch1, foff, iq = fixture_case(path)
    g = O.single_dm_geometry(nchans, x.shape[0], float(z["tsamp"]), fch1, foff, float(z["tstart"]),
                             float(z["tend"]), float(z["dm"]), float(z["freq_start"]),
                             float(z["freq_end"]), fil=fil)
    tsamp = float(z["tsamp"]) if fil else float(F32(z["tsamp"]))
    # mask-file channels index the data as read (a descending file already turned around)
    bad = z["bad"]
    spec, after = O.single_dm_with_rfi(x, nchans, g, tsamp, bool(z["use_mask"]), bad, iq)
    np.testing.assert_array_equal(spec, z["spec"])
    assert (F32(z["tstart"]), F32(g.tend), F32(g.freq_start), F32(g.freq_end)) == \
        tuple(z["meta"])
    if "zeroed" in z:
        np.testing.assert_array_equal(np.flatnonzero(after.reshape(-1) != x.reshape(-1)),
                                      z["zeroed"])


def _random_case(rng, it):
    nchans = int(rng.choice([16, 64, 100, 256]))
    ndata = int(rng.integers(500, 5000))
    tsamp = float(rng.choice([6.4e-5, 1e-4, 4.9152e-5, 1e-3]))
    fch1, foff = float(rng.uniform(300, 1400)), float(rng.uniform(0.05, 2.0))
    top = fch1 + (nchans - 1) * foff
    fs = float(rng.uniform(fch1 - 5, fch1 + 0.4 * (top - fch1)))
    fe = float(rng.uniform(fs + 0.2 * (top - fs), top + 3))
    T = ndata * tsamp
    ts = float(rng.uniform(0, 0.7 * T))
    te = float(ts + rng.uniform(-0.01, 0.5) * T)
    dm = float(rng.uniform(-5, 300))
    return dict(fil=bool(it % 2), nbits=int(rng.choice([8, 16, 32])), nchans=nchans, ndata=ndata,
                tsamp=tsamp, fch1=fch1, foff=foff, ts=ts, te=te, dm=dm, fs=fs, fe=fe)


def _oracle(c):
    try:
        return O.single_dm_geometry(c["nchans"], c["ndata"], c["tsamp"], c["fch1"], c["foff"],
                                    c["ts"], c["te"], c["dm"], c["fs"], c["fe"], fil=c["fil"])
    except ValueError as e:
        return e


@pytest.mark.skipif(not O.ref_gpu_available(32), reason="reference build absent")
def test_oracle_matches_reference_sweep():
    rng = np.random.default_rng(11)
    checked = errors = 0
    for it in range(60):
        c = _random_case(rng, it)
        if c["fil"] and c["dm"] < 0:
            continue   # the reference reads before the file for negative delays
        dt = {8: np.uint8, 16: np.uint16, 32: np.uint32}[c["nbits"]]
        x = rng.integers(0, 200, (c["ndata"], c["nchans"])).astype(dt)
        g = _oracle(c)
        try:
            if c["fil"]:
                with tempfile.TemporaryDirectory() as d:
                    p = os.path.join(d, "a.fil")
                    write_fil(p, x, c["tsamp"], c["fch1"], c["foff"])
                    r, meta = O.ref_gpu_fil_with_dm(p, c["nbits"], c["ts"], c["te"], c["dm"],
                                                    c["fs"], c["fe"])
            else:
                r, meta, _ = O.ref_gpu_spec_with_dm(x, c["nchans"], c["tsamp"], c["fch1"],
                                                    c["foff"], c["ts"], c["te"], c["dm"], c["fs"],
                                                    c["fe"])
        except ValueError as e:
            assert isinstance(g, ValueError), (it, c, e)
            errors += 1
            continue
        assert not isinstance(g, ValueError), (it, c, g)
        np.testing.assert_array_equal(O.single_dm_spectrum(x, c["nchans"], g), r)
        assert (F32(c["ts"]), F32(g.tend), F32(g.freq_start), F32(g.freq_end)) == tuple(meta)
        checked += 1
    assert checked >= 20 and errors >= 3


def test_library_geometry_matches_oracle():
    from astroflow_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(5)
    ok = bad = 0
    for it in range(300):
        c = _random_case(rng, it)
        g = _oracle(c)
        h = _lib.Header(0.0, c["tsamp"], c["fch1"], c["foff"], c["nbits"], c["nchans"], c["ndata"])
        q = _lib.SingleDmParams(c["ts"], c["te"], c["dm"], c["fs"], c["fe"],
                                _lib.FREQ_FIL if c["fil"] else _lib.FREQ_HEADER, None)
        info = _lib.SingleDmInfo()
        rc = L.dd_single_dm_geometry(ctypes.byref(h), ctypes.byref(q), ctypes.byref(info))
        if isinstance(g, ValueError):
            assert rc == _lib.DD_ERR_INVALID, (it, c, g)
            bad += 1
            continue
        assert rc == 0, (it, c, L.dd_last_error())
        got = (info.t_start, info.ntimes, info.chan_start, info.nchans, info.rfi_t0, info.rfi_len,
               F32(info.tend), F32(info.freq_start), F32(info.freq_end))
        want = (g.t_start, g.ntimes, g.chan_start, g.nchans, g.rfi_t0, g.rfi_len, F32(g.tend),
                F32(g.freq_start), F32(g.freq_end))
        assert got == want, (it, c)
        ok += 1
    assert ok >= 100 and bad >= 20


def test_library_geometry_errors():
    from astroflow_b200 import _lib
    L = _lib.load()
    h = _lib.Header(0.0, 1e-3, 1000.0, 1.0, 8, 64, 4096)
    cases = [((0.5, 0.5, 10.0, 1010.0, 1050.0), "tend must be > tstart"),
             ((5.0, 6.0, 10.0, 1010.0, 1050.0), "Invalid time window"),
             ((0.5, 1.0, -1.0, 1010.0, 1050.0), "dm must be >= 0"),
             ((0.5, 1.0, 10.0, 1050.0, 1010.0), "freq_end must be > freq_start"),
             ((0.5, 1.0, 10.0, 990.0, 1050.0), "out of file range"),
             ((3.9, 4.0, 3000.0, 1000.0, 1063.0), "Time window too short")]
    for (ts, te, dm, fs, fe), msg in cases:
        q = _lib.SingleDmParams(ts, te, dm, fs, fe, _lib.FREQ_HEADER, None)
        info = _lib.SingleDmInfo()
        assert L.dd_single_dm_geometry(ctypes.byref(h), ctypes.byref(q),
                                       ctypes.byref(info)) == _lib.DD_ERR_INVALID
        assert msg in L.dd_last_error().decode()
    # a Filterbank with descending frequencies is fine (the reader turned it around),
    # a Header with foff < 0 is refused like the reference does
    h2 = _lib.Header(0.0, 1e-3, 1063.0, -1.0, 8, 64, 4096)
    q = _lib.SingleDmParams(0.5, 1.0, 10.0, 1010.0, 1050.0, _lib.FREQ_HEADER, None)
    assert L.dd_single_dm_geometry(ctypes.byref(h2), ctypes.byref(q),
                                   ctypes.byref(_lib.SingleDmInfo())) == _lib.DD_ERR_INVALID
    assert "descending" in L.dd_last_error().decode()


@pytest.mark.skipif(not O.ref_gpu_available(32), reason="reference build absent")
@pytest.mark.parametrize("fil", [False, True], ids=["header", "filterbank"])
def test_library_errors_are_the_reference_messages(fil, tmp_path):
    """Rejected windows, bands and DMs: dd_single_dm_geometry (host code) fails where
    the reference's cpucal functions throw, with the same message word for word
    (include/cpucal.hpp:214-235, 282-284, 350-388, 430-432), and accepts what
    they accept."""
    from astroflow_b200 import _lib

    L = _lib.load()
    nchans, ndata, tsamp, fch1, foff = 64, 2000, 1e-3, 1200.0, 1.0
    x = np.random.default_rng(0).integers(0, 200, (ndata, nchans)).astype(np.uint8)
    path = str(tmp_path / "a.fil")
    write_fil(path, x, tsamp, fch1, foff)
    cases = [(0.5, 0.5, 10.0, 1200.0, 1250.0), (2.5, 3.0, 10.0, 1200.0, 1250.0),
             (0.1, 0.5, 10.0, 1250.0, 1250.0), (0.1, 0.5, -1.0, 1200.0, 1250.0),
             (0.1, 0.5, 10.0, 1100.0, 1250.0), (0.1, 0.5, 10.0, 1200.0, 1300.0),
             (1.99, 1.995, 500.0, 1200.0, 1263.0), (0.1, 0.5, 10.0, 1200.2, 1200.4)]
    rejected = 0
    for ts, te, dm, fs, fe in cases:
        try:
            if fil:
                O.ref_gpu_fil_with_dm(path, 8, ts, te, dm, fs, fe)
            else:
                O.ref_gpu_spec_with_dm(x, nchans, tsamp, fch1, foff, ts, te, dm, fs, fe)
            ref = None
        except ValueError as e:
            ref = str(e)
        h = _lib.Header(0.0, tsamp, fch1, foff, 8, nchans, ndata)
        q = _lib.SingleDmParams(ts, te, dm, fs, fe, _lib.FREQ_FIL if fil else _lib.FREQ_HEADER,
                                None)
        info = _lib.SingleDmInfo()
        rc = L.dd_single_dm_geometry(ctypes.byref(h), ctypes.byref(q), ctypes.byref(info))
        ours = None if rc == 0 else L.dd_last_error().decode()
        assert ours == ref, ((ts, te, dm, fs, fe), ours, ref)
        if rc:
            assert rc == _lib.DD_ERR_INVALID
            rejected += 1
    assert rejected >= 6
