"""The drop-in module astroflow_b200._astroflow_core on the GPU, against the
reference's own code run on the same GPU (oracle/_ref/libref_gpu_sb<W>.so):

  * _dedisperse_spec (src/bindpy/bindings.cpp:43-57 -> gpucal::dedisperse_spec<T>):
    the reference's raw sums, cut and imaged by the same image step
    (include/data.h:620-727), must give the same 512x512x3 images byte for byte;
  * _dedispered_fil target 1 (Filterbank reader + dedispered_fil_cuda<T>), same check;
  * _dedispered_fil target 0 (cpucal::dedispered_fil_omp semantics) against the
    oracle's brute force, slice by slice.
"""
import numpy as np
import pytest

from oracle import cv2_images as CVI
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
pytest.importorskip("cv2")
from astroflow_b200 import _astroflow_core as C  # noqa: E402
from astroflow_b200 import postprocess  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402
from sigproc_writer import write_fil  # noqa: E402

F32 = np.float32
W = C.SUBBAND_WIDTH


def need_ref():
    if not O.ref_gpu_available(W):
        pytest.skip("reference GPU build absent")


def chunk(nchans, n, nbits, tsamp, seed, rfi=0.0, impulses=0):
    spec = ChunkSpec(nchans=nchans, nsamp=n, nbits=nbits, tsamp=tsamp, seed=seed, rfi_frac=rfi,
                     rfi_amp=60.0 if nbits == 8 else 6000.0, impulses=impulses,
                     imp_amp=50.0 if nbits == 8 else 5000.0,
                     pulses=[(120.0, 0.3 * n * tsamp, 3 * tsamp, 40.0 if nbits == 8 else 4000.0)])
    x, _ = make_chunk(spec)
    return x, spec


def assert_same_images(got, want):
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert a.shape == (512, 512, 3) and a.dtype == np.uint8
        assert np.array_equal(a, b)


SPEC = [
    # nchans, N, nbits, tsamp, dm (lo, hi, step), ds, t_sample, rfi (mask, zdm, iqrm)
    (256, 8192, 8, 64e-6, (0.0, 300.0, 1.0), 1, 0.1, (True, True, True)),
    (256, 6000, 16, 64e-6, (5.0, 400.0, 0.5), 2, 0.07, (True, False, True)),
    (128, 4096, 32, 1e-4, (0.0, 200.0, 1.0), 1, 0.12, (False, False, False)),
]


@pytest.mark.parametrize("case", SPEC)
def test_dedisperse_spec_images_match_reference(case, tmp_path):
    need_ref()
    nchans, n, nbits, tsamp, (lo, hi, step), ds, tslice, (um, uz, ui) = case
    x, spec = chunk(nchans, n, nbits, tsamp, seed=5, rfi=0.05, impulses=3)
    mask = tmp_path / "mask.txt"
    mask.write_text("3 17 40\n100\n")
    hdr = C.Header(0.0, spec.tsamp, spec.fch1, spec.foff, nbits, nchans, n, "chunk")
    freq = O.freq_table_header(hdr.fch1, hdr.foff, nchans)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    iq = C.IQRMconfig(0, 0.05, 3.0, 1.5, 0.0, 0.0, True)
    rfi = C.RFIconfig(um, uz, ui, iq)
    res = C._dedisperse_spec(x, hdr, lo, hi, fs, fe, step, ds, tslice, 0, str(mask), rfi)
    ref = O.ref_gpu_dedisperse_spec(x, nchans, hdr.tsamp, hdr.fch1, hdr.foff, lo, hi, fs, fe, step,
                                    ds, tslice, sb_width=W, mask_file=str(mask), use_mask=um,
                                    use_zero_dm=uz, use_iqrm=ui, iq=iq)
    tsamp_out = float(F32(F32(hdr.tsamp) * F32(ds)))
    assert_same_images(res.dm_times, CVI.slice_images(ref, tsamp_out, 1, tslice))
    assert res.shape == [512, 512, 3] and res.dm_ndata == 512 and res.downtsample_ndata == 512
    assert (res.dm_low, res.dm_high, res.dm_step) == (float(F32(lo)), float(F32(hi)), float(F32(step)))
    assert res.tsample == float(F32(tslice)) and res.filname == "chunk"


def test_dedisperse_spec_accepts_3d_input():
    x, spec = chunk(128, 4096, 8, 64e-6, seed=9)
    hdr = C.Header(0.0, spec.tsamp, spec.fch1, spec.foff, 8, 128, 4096, "c")
    fs, fe = float(F32(hdr.fch1)), 1500.0
    a = C._dedisperse_spec(x, hdr, 0, 100, fs, fe, 1, 1, 0.05)
    b = C._dedisperse_spec(x.reshape(2048, 2, 128), hdr, 0, 100, fs, fe, 1, 1, 0.05)
    assert_same_images(a.dm_times, b.dm_times)


def test_dedisperse_spec_rejects_band_outside_header():
    """A band outside the header's raises ValueError with the reference's message
    (src/core/dedispered.cu:1009-1015), word for word against the reference build."""
    x, spec = chunk(64, 2048, 8, 64e-6, seed=1)
    hdr = C.Header(0.0, spec.tsamp, spec.fch1, spec.foff, 8, 64, 2048, "c")
    with pytest.raises(ValueError) as ours:
        C._dedisperse_spec(x, hdr, 0, 100, 900.0, 1500.0, 1, 1, 0.05)
    assert str(ours.value).startswith(
        "Frequency range [900.000-1500.000 MHz] out of spectrum range [")
    if O.ref_gpu_available(32):
        with pytest.raises(ValueError) as ref:
            O.ref_gpu_dedisperse_spec(x, 64, hdr.tsamp, hdr.fch1, hdr.foff, 0.0, 100.0, 900.0,
                                      1500.0, 1.0, 1, 0.05)
        assert str(ref.value).endswith(str(ours.value)), (str(ref.value), str(ours.value))


def test_dedispered_fil_rejects_band_outside_the_file(tmp_path):
    """The same for a file (src/core/dedispered.cu:483-986 through the Filterbank
    path): ValueError with the reference's message."""
    x, spec = chunk(64, 2048, 8, 64e-6, seed=2)
    path = tmp_path / "band.fil"
    write_fil(path, x, 64e-6, spec.fch1, spec.foff)
    fe = float(spec.fch1 + 63 * spec.foff)
    with pytest.raises(ValueError) as ours:
        C._dedispered_fil(str(path), 0.0, 100.0, 900.0, fe, 1.0, 1, 0.05, 1, 0)
    assert str(ours.value).startswith("Frequency range [900.000-")
    if O.ref_gpu_available(32):
        with pytest.raises(ValueError) as ref:
            O.ref_gpu_dedispered_fil(path, 0.0, 100.0, 900.0, fe, 1.0, 1, 0.05)
        assert str(ref.value).endswith(str(ours.value)), (str(ref.value), str(ours.value))


FIL = [
    # nchans, N, nbits, tsamp, descending, dm (lo, hi, step), ds, t_sample, rfi (mask, zdm, iqrm)
    (192, 5000, 8, 64e-6, True, (0.0, 250.0, 1.0), 1, 0.1, (False, True, True)),
    (128, 4000, 16, 1e-4, False, (0.0, 300.0, 2.0), 2, 0.15, (True, False, False)),
]


@pytest.mark.parametrize("case", FIL)
def test_dedispered_fil_gpu_images_match_reference(case, tmp_path):
    need_ref()
    nchans, n, nbits, tsamp, desc, (lo, hi, step), ds, tslice, (um, uz, ui) = case
    x, spec = chunk(nchans, n, nbits, tsamp, seed=11, rfi=0.04, impulses=2)
    path = tmp_path / "obs.fil"
    if desc:
        write_fil(path, x[:, ::-1], tsamp, spec.f_hi, -spec.foff)
    else:
        write_fil(path, x, tsamp, spec.fch1, spec.foff)
    mask = tmp_path / "mask.txt"
    mask.write_text("5 6 7 8\n")
    fil = C.Filterbank(str(path))
    fs, fe = float(F32(fil.frequency_table[2])), float(F32(fil.frequency_table[-3]))
    iq = C.IQRMconfig(1, 0.05, 3.0, 1.5, 0.0, 0.0, True)
    rfi = C.RFIconfig(um, uz, ui, iq)
    res = C._dedispered_fil(str(path), lo, hi, fs, fe, step, ds, tslice, 1, 0, str(mask), rfi)
    ref = O.ref_gpu_dedispered_fil(path, lo, hi, fs, fe, step, ds, tslice, sb_width=W,
                                   mask_file=str(mask), use_mask=um, use_zero_dm=uz,
                                   use_iqrm=ui, iq=iq)
    tsamp_out = float(F32(tsamp * ds))
    assert_same_images(res.dm_times, CVI.slice_images(ref, tsamp_out, 1, tslice))


def test_dedispered_fil_cpu_target_matches_oracle(tmp_path):
    nchans, n, tsamp = 96, 3000, 64e-6
    x, spec = chunk(nchans, n, 8, tsamp, seed=13)
    path = tmp_path / "cpu.fil"
    write_fil(path, x[:, ::-1], tsamp, spec.f_hi, -spec.foff)
    fil = C.Filterbank(str(path))
    fs, fe = float(fil.frequency_table[0]), float(fil.frequency_table[-1])
    lo, hi, step, ds, tslice = 0.0, 200.0, 1.0, 2, 0.05
    res = C._dedispered_fil(str(path), lo, hi, fs, fe, step, ds, tslice, 0)
    # the oracle's sums with the delay table of the reference CPU build's arithmetic
    # (the library's default; the table itself is pinned by tests/test_brute_table_cpu.py)
    from astroflow_b200.dedisp import brute_delay_table
    freq = np.asarray(fil.frequency_table, np.float64)
    cs, ce = O.chan_range(freq, fs, fe)
    table, _ = brute_delay_table(freq, cs, ce, ce, lo, step, O.dm_steps(lo, hi, step), fil.tsamp)
    slices = O.bruteforce_cpu(fil.data.reshape(n, nchans), nchans, fil.frequency_table, fil.tsamp,
                              lo, hi, fs, fe, step, ds, tslice, delay=table)
    assert_same_images(res.dm_times, CVI.images(slices))


def test_filterbank_path_matches_reference_on_random_files(tmp_path):
    """SIGPROC files with seeded random channel counts, band edges, channel order and
    DM grids, read straight to the device (ingest.read_filterbank) and dedispersed
    with the file's frequency table: the raw DM-time sums equal the reference's
    file entry point (Filterbank + dedispered_fil_cuda) bit for bit."""
    need_ref()
    from astroflow_b200 import ingest
    from astroflow_b200.dedisp import Plan

    rng = np.random.default_rng(77)
    checked = 0
    for it in range(8):
        nchans = int(rng.choice([96, 254, 300, 512]))
        n = int(rng.integers(3000, 9000))
        tsamp = float(rng.choice([49.152e-6, 64e-6, 1e-4]))
        foff = float(rng.uniform(0.3, 2.0)) * (1 if it % 2 else -1)
        fch1 = float(rng.uniform(1100, 1500))
        raw = rng.integers(0, 200, (n, nchans), dtype=np.uint8)
        p = str(tmp_path / f"r{it}.fil")
        write_fil(p, raw, tsamp, fch1, foff)
        x, h, table = ingest.read_filterbank(p)
        fs, fe = float(F32(table[int(0.05 * nchans)])), float(F32(table[-1 - int(0.1 * nchans)]))
        lo, hi, step, ds = 0.0, float(rng.uniform(80, 400)), float(rng.choice([0.5, 1.0])), int(rng.choice([1, 2]))
        ref = O.ref_gpu_dedispered_fil(p, lo, hi, fs, fe, step, ds, 0.5, sb_width=W, cap=1 << 24)
        hdr = dict(tsamp=h["tsamp"], fch1=h["fch1"], foff=h["foff"], nbits=8, nchans=nchans, ndata=n)
        plan = Plan(hdr, lo, hi, fs, fe, step, ds, algorithm="subband", subband_width=W,
                    zero_dm_mode=C.ZERO_DM_MODE, freq_mode="fil", freq_table=table)
        out = plan.run(x.view(-1))
        got = out.view(torch.int32).cpu().numpy().view(np.uint32)
        plan.close()
        assert got.shape == ref.shape
        np.testing.assert_array_equal(got, ref, err_msg=f"file {it}")
        checked += 1
    assert checked == 8
