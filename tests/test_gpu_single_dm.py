"""Single-DM dedispersed spectra on the GPU (dd_single_dm_run and the drop-in
_dedisperse_spec_with_dm / _dedispered_fil_with_dm_uint{8,16,32},
src/bindpy/bindings.cpp:31-42, 59-67 -> include/cpucal.hpp:203-483):

  * against the reference's golden fixtures (spectrum, tstart/tend/band, and the
    samples the reference zeroes in the caller's array);
  * against the reference itself run here (oracle/_ref/libref_gpu_sb32.so), over
    seeded random windows, DMs, bands, sample widths, mask files and IQRM settings;
  * the binding's argument order and its in-place masking of the caller's array.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200 import _astroflow_core as C  # noqa: E402
from astroflow_b200.dedisp import IqrmParams, RfiParams, single_dm_spectrum  # noqa: E402
from sigproc_writer import write_fil  # noqa: E402
from test_single_dm_cpu import FIXTURES, fixture_case  # noqa: E402

F32 = np.float32
DT = {8: np.uint8, 16: np.uint16, 32: np.uint32}


def _rficfg(use_mask, iq):
    if iq is None:
        return C.RFIconfig(bool(use_mask), False, False, C.IQRMconfig())
    return C.RFIconfig(bool(use_mask), False, True,
                       C.IQRMconfig(int(iq[0]), iq[1], iq[2], 1.5, iq[3], iq[4], True))


def _mask_file(tmp_path, bad):
    p = tmp_path / "mask.txt"
    p.write_text(" ".join(str(int(b)) for b in bad) + "\n")
    return str(p)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[11:-4] for p in FIXTURES])
def test_golden(path, tmp_path):
    z, x, nchans, fil, fch1, foff, _ = fixture_case(path)
    iq = z["iq"] if z["iq"].size else None
    mask = _mask_file(tmp_path, z["bad"])
    args = (float(z["tstart"]), float(z["tend"]), float(z["dm"]), float(z["freq_start"]),
            float(z["freq_end"]), mask, _rficfg(bool(z["use_mask"]), iq))
    if fil:
        raw = z["data"]
        p = str(tmp_path / "a.fil")
        write_fil(p, raw, float(z["tsamp"]), float(z["fch1"]), float(z["foff"]))
        fb = C.Filterbank(p)
        s = getattr(C, f"_dedispered_fil_with_dm_uint{raw.dtype.itemsize * 8}")(fb, *args)
    else:
        hdr = C.Header(0.0, float(z["tsamp"]), fch1, foff, x.dtype.itemsize * 8, nchans,
                       x.shape[0], "golden")
        a = x.copy()
        ts, te, dm = args[:3]
        s = C._dedisperse_spec_with_dm(a, hdr, ts, te, dm, *args[3:])   # positional: tend, dm
        np.testing.assert_array_equal(np.flatnonzero(a.reshape(-1) != x.reshape(-1)),
                                      z["zeroed"])
    np.testing.assert_array_equal(s.data, z["spec"])
    assert (s.ntimes, s.nchans) == z["spec"].shape
    assert (F32(s.tstart), F32(s.tend), F32(s.freq_start), F32(s.freq_end)) == tuple(z["meta"])
    assert s.dm == F32(z["dm"])


def need_ref():
    if not O.ref_gpu_available(32):
        pytest.skip("reference GPU build absent")


def _case(rng, it):
    nchans = int(rng.choice([32, 64, 100, 256, 1024]))
    ndata = int(rng.integers(2000, 12000))
    tsamp = float(F32(rng.choice([6.4e-5, 1e-4, 4.9152e-5, 2.5e-4])))
    fch1, foff = float(F32(rng.uniform(300, 1400))), float(F32(rng.uniform(0.1, 1.5)))
    top = fch1 + (nchans - 1) * foff
    fs = float(rng.uniform(fch1, fch1 + 0.3 * (top - fch1)))
    fe = float(rng.uniform(fs + 0.3 * (top - fs), top))
    T = ndata * tsamp
    ts = float(rng.uniform(0, 0.5 * T))
    te = float(ts + rng.uniform(0.05, 0.5) * T)
    nbits = int(rng.choice([8, 16, 32]))
    hi = {8: 255, 16: 65535, 32: 1 << 24}[nbits]
    x = rng.normal(0.5 * hi, 0.08 * hi, size=(ndata, nchans))
    x[:, rng.choice(nchans, size=max(1, nchans // 16), replace=False)] += 0.3 * hi
    x = np.clip(np.rint(x), 0, hi).astype(DT[nbits])
    dm_max = 0.8 * ts / (4148.808 * (1 / fs ** 2 - 1 / fe ** 2)) if ts > 0 else 50.0
    dm = float(rng.uniform(0, max(1.0, min(dm_max, 400.0))))
    iq = None
    if it % 3:
        iq = (int(rng.integers(0, 2)), float(rng.uniform(0.05, 0.15)), float(rng.uniform(2, 4)),
              float(rng.choice([0.0, 0.2 * T])), float(rng.choice([0.0, 0.1 * T])))
    return dict(x=x, nchans=nchans, tsamp=tsamp, fch1=fch1, foff=foff, ts=ts, te=te, dm=dm,
                fs=fs, fe=fe, nbits=nbits, use_mask=bool(it % 2), iq=iq,
                bad=sorted(int(c) for c in rng.choice(nchans, size=5, replace=False)))


@pytest.mark.parametrize("fil", [False, True], ids=["header", "fil"])
def test_matches_reference_sweep(fil, tmp_path):
    need_ref()
    rng = np.random.default_rng(21 + fil)
    done = 0
    for it in range(24):
        c = _case(rng, it)
        mask = _mask_file(tmp_path, c["bad"])
        iqo = None
        if c["iq"] is not None:
            m, rf, ns, ws, hs = c["iq"]
            iqo = type("Iq", (), dict(mode=m, radius_frac=rf, nsigma=ns, geofactor=1.5,
                                      win_sec=ws, hop_sec=hs, include_tail=True))()
        cfg = _rficfg(c["use_mask"], c["iq"])
        try:
            if fil:
                p = str(tmp_path / f"c{it}.fil")
                write_fil(p, c["x"], c["tsamp"], c["fch1"], c["foff"])
                want, meta = O.ref_gpu_fil_with_dm(p, c["nbits"], c["ts"], c["te"], c["dm"],
                                                   c["fs"], c["fe"], mask, use_mask=c["use_mask"],
                                                   use_iqrm=iqo is not None, iq=iqo)
            else:
                want, meta, after = O.ref_gpu_spec_with_dm(
                    c["x"], c["nchans"], c["tsamp"], c["fch1"], c["foff"], c["ts"], c["te"],
                    c["dm"], c["fs"], c["fe"], mask, use_mask=c["use_mask"],
                    use_iqrm=iqo is not None, iq=iqo)
        except ValueError as e:
            with pytest.raises(ValueError):
                if fil:
                    getattr(C, f"_dedispered_fil_with_dm_uint{c['nbits']}")(
                        C.Filterbank(p), c["ts"], c["te"], c["dm"], c["fs"], c["fe"], mask, cfg)
                else:
                    hdr = C.Header(0.0, c["tsamp"], c["fch1"], c["foff"], c["nbits"],
                                   c["nchans"], c["x"].shape[0], "sweep")
                    C._dedisperse_spec_with_dm(c["x"].copy(), hdr, c["ts"], c["te"], c["dm"],
                                               c["fs"], c["fe"], mask, cfg)
            continue
        if fil:
            fb = C.Filterbank(p)
            s = getattr(C, f"_dedispered_fil_with_dm_uint{c['nbits']}")(
                fb, c["ts"], c["te"], c["dm"], c["fs"], c["fe"], mask, cfg)
        else:
            hdr = C.Header(0.0, c["tsamp"], c["fch1"], c["foff"], c["nbits"], c["nchans"],
                           c["x"].shape[0], "sweep")
            a = c["x"].copy()
            s = C._dedisperse_spec_with_dm(a, hdr, c["ts"], c["te"], c["dm"], c["fs"], c["fe"],
                                           mask, cfg)
            np.testing.assert_array_equal(a, after, err_msg=f"case {it}: caller's array")
        np.testing.assert_array_equal(s.data, want, err_msg=f"case {it}")
        assert (F32(s.tstart), F32(s.tend), F32(s.freq_start), F32(s.freq_end)) == tuple(meta)
        done += 1
    assert done >= 12


def test_binding_argument_order():
    """The binding names its 4th/5th parameters dm/tend while the function takes
    tend/dm (pyapi.cpp:330-332 vs bindings.cpp:59-61): keywords follow the names."""
    rng = np.random.default_rng(3)
    x = rng.integers(0, 255, (4000, 64), dtype=np.uint8)
    hdr = C.Header(0.0, 1e-4, 1200.0, 1.0, 8, 64, 4000, "args")
    cfg = C.RFIconfig()
    a = C._dedisperse_spec_with_dm(x, hdr, 0.05, 0.2, 30.0, 1210.0, 1260.0, "", cfg)
    b = C._dedisperse_spec_with_dm(x, hdr, 0.05, dm=0.2, tend=30.0, freq_start=1210.0,
                                   freq_end=1260.0, maskfile="", rficfg=cfg)
    assert a.dm == b.dm == F32(30.0) and a.tend == b.tend
    np.testing.assert_array_equal(a.data, b.data)
    assert isinstance(a, C.Spectrum8) and a.nbits == 8
    g = O.single_dm_geometry(64, 4000, 1e-4, 1200.0, 1.0, 0.05, 0.2, 30.0, 1210.0, 1260.0)
    np.testing.assert_array_equal(a.data, O.single_dm_spectrum(x, 64, g))


def test_device_api_masked_rows():
    """dd_single_dm_run leaves its input alone and reports the processed rows."""
    rng = np.random.default_rng(9)
    x = rng.integers(0, 60000, (6000, 128)).astype(np.uint16)
    x[:, 7] = 65000
    hdr = dict(tsamp=1e-4, fch1=1100.0, foff=2.0, nbits=16, nchans=128, ndata=6000)
    xd = torch.from_numpy(x.view(np.int16)).cuda().view(torch.uint16)
    before = xd.clone()
    rfi = RfiParams(use_mask=True, use_iqrm=True, iqrm=IqrmParams(0, 0.1, 3.0, 1.5, 0.1, 0.05, True))
    spec, g, rows = single_dm_spectrum(xd, hdr, 0.1, 0.4, 80.0, 1105.0, 1300.0, rfi=rfi,
                                       bad_channels=[3, 50], masked_rows=True)
    torch.cuda.synchronize()
    assert torch.equal(xd, before)
    rows = rows.view(torch.int16).cpu().numpy().view(np.uint16)
    assert rows.shape == (g["rfi_len"], 128)
    assert (rows[:, 3] == 0).all() and (rows[:, 50] == 0).all()
    geo = O.single_dm_geometry(128, 6000, 1e-4, 1100.0, 2.0, 0.1, 0.4, 80.0, 1105.0, 1300.0)
    x2 = x.copy()
    x2[g["rfi_t0"]:g["rfi_t0"] + g["rfi_len"]] = rows
    np.testing.assert_array_equal(spec.view(torch.int16).cpu().numpy().view(np.uint16),
                                  O.single_dm_spectrum(x2, 128, geo))


@pytest.mark.parametrize("nbits", [8, 16, 32])
def test_dm_zero_is_the_channel_slice(nbits, tmp_path):
    """The reference's own known answer (python/tests/test_dedispered.py:21-101): at
    DM 0 the spectrum is the raw channel slice of the window, for a descending
    Filterbank after the reader has turned it around."""
    rng = np.random.default_rng(nbits)
    raw = rng.integers(0, 250, (3000, 96)).astype(DT[nbits])
    p = str(tmp_path / "d.fil")
    write_fil(p, raw, 64e-6, 1500.0, -2.0)
    fb = C.Filterbank(p)
    f = getattr(C, f"_dedispered_fil_with_dm_uint{nbits}")
    fs, fe = float(fb.frequency_table[0]), float(fb.frequency_table[-1])
    s = f(fb, 0.0, 0.1, 0.0, fs, fe, "", C.RFIconfig())
    n = int(0.1 / 64e-6)
    assert s.data.shape == (n, 96) and (s.freq_start, s.freq_end) == (F32(fs), F32(fe))
    np.testing.assert_array_equal(s.data, raw[:n, ::-1])
    hdr = C.Header(0.0, 64e-6, 1100.0, 2.0, nbits, 96, 3000, "h")
    s = C._dedisperse_spec_with_dm(raw, hdr, 0.0, 3000 * 64e-6, 0.0, 1150.0, 1250.0, "",
                                   C.RFIconfig())
    cs, ce = 25, 75   # (f - fch1) / foff at the band edges, both inclusive
    np.testing.assert_array_equal(s.data, raw[:s.ntimes, cs:ce + 1])
