"""GPU parity of the dedispersion path against the oracle and the reference's own code.

Ground truth:
  * oracle/liboracle.so — the CPU restatement (oracle/dd_oracle.c);
  * oracle/_ref/libref_cpu.so — the reference's CPU brute force (include/cpucal.hpp)
    compiled from its sources;
  * oracle/_ref/libref_gpu_sb<W>.so — the reference's GPU path (src/core/dedispered.cu,
    src/core/iqrm.cu, src/rfi/rfimarker.cu) compiled for sm_100a, run on this GPU.
Integer outputs, delay tables and masks must match bit for bit.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import IqrmParams, Plan, RfiParams  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


def to_np(t):
    if t.dtype == torch.uint32:
        return t.view(torch.int32).cpu().numpy().view(np.uint32)
    if t.dtype == torch.uint64:
        return t.view(torch.int64).cpu().numpy().view(np.uint64)
    if t.dtype == torch.uint16:
        return t.view(torch.int16).cpu().numpy().view(np.uint16)
    return t.cpu().numpy()


def dev(x):
    x = np.ascontiguousarray(x)
    if x.dtype == np.uint16:
        return torch.from_numpy(x.view(np.int16)).cuda().view(torch.uint16)
    if x.dtype == np.uint32:
        return torch.from_numpy(x.view(np.int32)).cuda().view(torch.uint32)
    return torch.from_numpy(x).cuda()


def rand_data(rng, n, nchans, nbits):
    hi = {8: 256, 16: 65536, 32: 1 << 20}[nbits]
    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32}[nbits]
    return rng.integers(0, hi, size=(n, nchans)).astype(dt)


# ------------------------------------------------------------------ brute force
BRUTE = [
    # nchans, N, nbits, tsamp, fch1, foff, dm_low, dm_high, dm_step, ds, t_sample
    (64, 4096, 8, 64e-6, 1000.0, 500 / 64, 0.0, 100.0, 1.0, 1, 0.1),
    (96, 3000, 8, 49.152e-6, 1200.0, 0.3, 0.0, 900.0, 0.3, 2, 0.05),
    (128, 2048, 16, 1e-4, 1100.1, 0.77, 10.0, 1200.0, 2.3, 3, 0.061),
    (50, 5000, 8, 1.26646875e-3, 1130.0, 1.0, 10.0, 600.0, 1.0, 1, 0.5),
    (33, 1500, 32, 64e-6, 1300.0, 2.0, 0.0, 300.0, 1.5, 1, 0.04),
    (300, 1024, 8, 64e-6, 1000.0, 1.6, 0.0, 50.0, 0.5, 4, 0.0655),
    # 16-bit samples through the staged 32-bit sums: 512 full-range channels, so the
    # whole-pair sum wraps many times before the low halves are recovered
    (512, 3000, 16, 64e-6, 1000.0, 0.9, 0.0, 200.0, 1.0, 1, 0.1),
]


@pytest.mark.parametrize("case", BRUTE)
def test_brute_force_matches_oracle(case):
    nchans, N, nbits, tsamp, fch1, foff, lo, hi, step, ds, tslice = case
    rng = np.random.default_rng(hash(case) & 0xFFFF)
    x = rand_data(rng, N, nchans, nbits)
    freq = O.freq_table_fil(fch1, foff, nchans)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    hdr = dict(tsamp=tsamp, fch1=fch1, foff=foff, nbits=nbits, nchans=nchans, ndata=N)
    # the oracle restates the table in IEEE arithmetic: compare with that mode
    plan = Plan(hdr, lo, hi, fs, fe, step, ds, tslice, algorithm="brute", freq_mode="fil",
                table_mode="ieee")
    out = to_np(plan.run(dev(x)))
    ref = np.concatenate(O.bruteforce_cpu(x, nchans, freq, tsamp, lo, hi, fs, fe, step, ds, tslice), axis=1)
    d, _ = plan.tables()
    cs, ce = O.chan_range(freq, fs, fe)
    assert np.array_equal(d, O.cpu_delay_table(freq, cs, ce, lo, step, d.shape[0], tsamp))
    assert out.shape == ref.shape
    assert np.array_equal(out, ref)


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
@pytest.mark.parametrize("case", BRUTE[:3])
def test_brute_force_matches_reference_cpu(case):
    """With the reference build's own delay table injected, the sums equal the
    reference's cpucal::dedispered_fil_omp bit for bit (its table itself depends
    on the host CPU's vector reciprocal at rounding ties)."""
    nchans, N, nbits, tsamp, fch1, foff, lo, hi, step, ds, tslice = case
    if nbits == 32:
        pytest.skip("probe uses 8-bit impulses")
    rng = np.random.default_rng(7)
    x = rand_data(rng, N, nchans, nbits)
    freq = O.freq_table_fil(fch1, foff, nchans)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    D = O.ref_cpu_delays(nchans, N, fch1, foff, tsamp, lo, hi, fs, fe, step)
    hdr = dict(tsamp=tsamp, fch1=fch1, foff=foff, nbits=nbits, nchans=nchans, ndata=N)
    plan = Plan(hdr, lo, hi, fs, fe, step, ds, tslice, algorithm="brute", freq_mode="fil")
    plan.set_delay_table(D)
    out = to_np(plan.run(dev(x)))
    ref = np.concatenate(O.ref_bruteforce_cpu(x, nchans, fch1, foff, tsamp, lo, hi, fs, fe, step, ds, tslice), axis=1)
    assert np.array_equal(out, ref)


# ------------------------------------------------------------------ subband
SUB = [
    # nchans, N, nbits, tsamp, f_hi, bw, dm_low, dm_high, dm_step, ds, sbw, band
    (256, 8192, 8, 49.152e-6, 1500.0, 500.0, 0.0, 300.0, 1.0, 1, 32, None),
    (256, 6000, 8, 64e-6, 1450.0, 300.0, 5.0, 700.0, 0.5, 2, 64, None),
    (512, 4096, 16, 1e-4, 1500.0, 500.0, 0.0, 1000.0, 2.0, 1, 32, None),
    (200, 5000, 8, 49.152e-6, 1500.0, 400.0, 0.0, 200.0, 0.7, 3, 16, (0.2, 0.9)),
    (128, 3333, 8, 64e-6, 1400.0, 200.0, 0.0, 500.0, 1.0, 1, 64, (0.0, 0.5)),
    (256, 4096, 32, 64e-6, 1500.0, 400.0, 0.0, 400.0, 1.0, 1, 32, None),
    (96, 3000, 32, 1e-4, 1450.0, 300.0, 3.0, 600.0, 0.9, 2, 16, (0.1, 0.8)),
    # edges: channel counts off the 4-sample word (the layout kernels' general path),
    # an odd chunk length, a single DM trial, a chunk far shorter than the largest
    # delay with a binning tail, and a subband width that is not a power of two
    (251, 3001, 8, 49.152e-6, 1500.0, 400.0, 0.0, 150.0, 1.0, 1, 32, None),
    (250, 2048, 16, 1e-4, 1500.0, 500.0, 100.0, 100.0, 1.0, 1, 16, None),
    (97, 1501, 8, 64e-6, 1450.0, 300.0, 0.0, 2000.0, 5.0, 4, 16, None),
    (130, 2500, 8, 64e-6, 1400.0, 200.0, 0.0, 300.0, 1.0, 1, 20, (0.05, 0.95)),
]


def sub_setup(case, seed=0):
    nchans, N, nbits, tsamp, f_hi, bw, lo, hi, step, ds, sbw, band = case
    spec = ChunkSpec(nchans=nchans, nsamp=N, nbits=nbits, f_hi=f_hi, bandwidth=bw, tsamp=tsamp,
                     seed=seed, pulses=[(0.4 * hi + 3, 0.1 * N * tsamp, 4 * tsamp, 30.0)])
    x, _ = make_chunk(spec)
    tsamp32, fch1_32, foff32 = float(F32(tsamp)), float(F32(spec.fch1)), float(F32(spec.foff))
    freq = O.freq_table_header(fch1_32, foff32, nchans)
    if band is None:
        fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    else:
        fs = float(F32(freq[0] + band[0] * (freq[-1] - freq[0])))
        fe = float(F32(freq[0] + band[1] * (freq[-1] - freq[0])))
    hdr = dict(tsamp=tsamp32, fch1=fch1_32, foff=foff32, nbits=nbits, nchans=nchans, ndata=N)
    return x, hdr, freq, fs, fe


@pytest.mark.parametrize("case", SUB)
def test_subband_sums_match_oracle(case):
    nchans, N, nbits, tsamp, f_hi, bw, lo, hi, step, ds, sbw, band = case
    x, hdr, freq, fs, fe = sub_setup(case)
    plan = Plan(hdr, lo, hi, fs, fe, step, ds, algorithm="subband", subband_width=sbw)
    out = to_np(plan.run(dev(x)))
    d1, r2 = plan.tables()
    xb = O.time_binning(x, nchans, ds) if ds > 1 else x
    op = O.subband_plan(freq, N, lo, hi, fs, fe, step, ds, sb_width=sbw)
    assert (op.chan_start, op.chan_end, op.dm_steps) == (plan.info["chan_start"], plan.info["chan_end"], plan.info["dm_steps"])
    ref = O.subband_sums(xb, nchans, op, d1, r2)
    assert out.shape == ref.shape
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("case", SUB)
def test_subband_tables_match_reference_gpu(case):
    nchans, N, nbits, tsamp, f_hi, bw, lo, hi, step, ds, sbw, band = case
    if not O.ref_gpu_available(sbw):
        pytest.skip("reference GPU build absent")
    x, hdr, freq, fs, fe = sub_setup(case)
    d1_ref, r2_ref, info = O.ref_gpu_tables(nchans, N, hdr["tsamp"], hdr["fch1"], hdr["foff"], lo,
                                            hi, fs, fe, step, ds, sb_width=sbw)
    plan = Plan(hdr, lo, hi, fs, fe, step, ds, algorithm="subband", subband_width=sbw)
    d1, r2 = plan.tables()
    assert info["chan_start"] == plan.info["chan_start"] and info["chan_end"] == plan.info["chan_end"]
    assert np.array_equal(d1, d1_ref)
    assert np.array_equal(r2, r2_ref)


@pytest.mark.parametrize("case", SUB)
def test_subband_matches_reference_gpu_call(case):
    nchans, N, nbits, tsamp, f_hi, bw, lo, hi, step, ds, sbw, band = case
    if not O.ref_gpu_available(sbw):
        pytest.skip("reference GPU build absent")
    x, hdr, freq, fs, fe = sub_setup(case)
    ref = O.ref_gpu_dedisperse_spec(x, nchans, hdr["tsamp"], hdr["fch1"], hdr["foff"], lo, hi, fs,
                                    fe, step, ds, sb_width=sbw)
    plan = Plan(hdr, lo, hi, fs, fe, step, ds, algorithm="subband", subband_width=sbw)
    out = to_np(plan.run(dev(x)))
    assert out.shape == ref.shape
    assert np.array_equal(out, ref)


# ------------------------------------------------------------------ RFI stages
RFI = [
    # nchans, N, nbits, ds, band, iq (mode, radius_frac, nsigma, win_sec, hop_sec)
    (256, 8192, 8, 1, None, (0, 0.1, 3.0, 0.0, 0.5)),
    (256, 8192, 8, 2, None, (1, 0.1, 3.0, 0.0, 0.5)),
    (300, 6000, 8, 1, (0.1, 0.95), (1, 0.05, 2.5, 0.05, 0.03)),
    (512, 4096, 16, 1, None, (1, 0.02, 3.0, 0.0, 2.5)),
    (160, 9000, 8, 3, (0.3, 1.0), (0, 0.2, 4.0, 0.1, 0.1)),
    (301, 5001, 8, 1, None, (0, 0.1, 3.0, 0.0, 0.0)),
    (254, 4001, 16, 1, (0.0, 0.9), (1, 0.1, 3.0, 0.0, 0.0)),
]


def rfi_setup(case, seed=3):
    nchans, N, nbits, ds, band, iqp = case
    spec = ChunkSpec(nchans=nchans, nsamp=N, nbits=nbits, seed=seed, rfi_frac=0.05, impulses=6,
                     rfi_amp=60 if nbits == 8 else 6000, imp_amp=50 if nbits == 8 else 5000,
                     pulses=[(150.0, 0.05, 2e-4, 25.0 if nbits == 8 else 2500.0)])
    x, _ = make_chunk(spec)
    tsamp32, fch1_32, foff32 = float(F32(spec.tsamp)), float(F32(spec.fch1)), float(F32(spec.foff))
    freq = O.freq_table_header(fch1_32, foff32, nchans)
    if band is None:
        fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    else:
        fs = float(F32(freq[0] + band[0] * (freq[-1] - freq[0])))
        fe = float(F32(freq[0] + band[1] * (freq[-1] - freq[0])))
    hdr = dict(tsamp=tsamp32, fch1=fch1_32, foff=foff32, nbits=nbits, nchans=nchans, ndata=N)
    mode, rf, ns, win, hop = iqp
    iq = IqrmParams(mode=mode, radius_frac=rf, nsigma=ns, geofactor=1.5, win_sec=win, hop_sec=hop,
                    include_tail=True)
    return x, hdr, freq, fs, fe, iq


def run_prepped(plan, x, nchans):
    n_win = max(int(plan.info["n_iqrm_windows"]), 1)
    masks = torch.zeros((n_win, nchans), dtype=torch.uint8, device="cuda")
    bounds = torch.zeros((n_win, 2), dtype=torch.int32, device="cuda")
    nb = int(plan.info["nsamp_binned"])
    prepped = torch.zeros((nb, nchans), dtype=dev(x[:1]).dtype, device="cuda")
    out = plan.run(dev(x), iqrm_masks=masks, iqrm_bounds=bounds, prepped=prepped)
    return to_np(out), masks.cpu().numpy(), bounds.cpu().numpy().view(np.uint32), to_np(prepped)


@pytest.mark.parametrize("case", RFI)
def test_iqrm_and_rfi_pipeline_match_reference_gpu(case):
    nchans, N, nbits, ds, band, iqp = case
    if not O.ref_gpu_available(32):
        pytest.skip("reference GPU build absent")
    x, hdr, freq, fs, fe, iq = rfi_setup(case)
    bad = [3, 17, nchans - 5]
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as fh:
        fh.write(" ".join(str(b) for b in bad) + "\n")
        mask_file = fh.name
    try:
        ref_x, t0, t1, ref_masks = O.ref_gpu_rfi(x, nchans, hdr["tsamp"], hdr["fch1"], hdr["foff"], fs,
                                                 fe, ds, mask_file=mask_file, use_mask=True,
                                                 use_zero_dm=True, use_iqrm=True, iq=iq)
        ref_out = O.ref_gpu_dedisperse_spec(x, nchans, hdr["tsamp"], hdr["fch1"], hdr["foff"], 0.0,
                                            200.0, fs, fe, 1.0, ds, mask_file=mask_file,
                                            use_mask=True, use_zero_dm=True, use_iqrm=True, iq=iq)
    finally:
        os.unlink(mask_file)
    plan = Plan(hdr, 0.0, 200.0, fs, fe, 1.0, ds, algorithm="subband",
                rfi=RfiParams(use_mask=True, use_zero_dm=True, use_iqrm=True, iqrm=iq),
                bad_channels=bad)
    out, masks, bounds, prepped = run_prepped(plan, x, nchans)
    assert len(t0) == plan.info["n_iqrm_windows"]
    assert np.array_equal(bounds[:, 0], t0) and np.array_equal(bounds[:, 1], t1)
    assert np.array_equal(masks, ref_masks), f"IQRM masks differ in {int((masks != ref_masks).sum())} entries"
    assert np.array_equal(prepped, ref_x)
    assert np.array_equal(out, ref_out)


@pytest.mark.parametrize("case", RFI[:3])
def test_zero_dm_range_matches_oracle(case):
    nchans, N, nbits, ds, band, iqp = case
    x, hdr, freq, fs, fe, iq = rfi_setup(case)
    plan = Plan(hdr, 0.0, 100.0, fs, fe, 1.0, ds, algorithm="subband", zero_dm_mode="range",
                rfi=RfiParams(use_zero_dm=True, use_iqrm=True, iqrm=iq))
    out, masks, bounds, prepped = run_prepped(plan, x, nchans)
    xb = O.time_binning(x, nchans, ds) if ds > 1 else x.copy()
    cs, ce = plan.info["chan_start"], plan.info["chan_end"]
    t0, t1, om = O.iqrm_masks(xb, nchans, cs, ce, float(F32(F32(hdr["tsamp"]) * F32(ds))), iq)
    assert np.array_equal(om, masks), "oracle IQRM masks differ"
    O.apply_window_masks(xb, nchans, t0, t1, om)
    O.zero_dm_range_exact(xb, nchans, cs, ce)
    assert np.array_equal(prepped, xb)


def test_time_binning_matches_oracle():
    rng = np.random.default_rng(5)
    for nbits in (8, 16):
        for ds in (2, 3, 8):
            x = rand_data(rng, 1003, 96, nbits)
            hdr = dict(tsamp=6.4e-5, fch1=1000.0, foff=1.0, nbits=nbits, nchans=96, ndata=1003)
            plan = Plan(hdr, 0.0, 10.0, 1000.0, 1095.0, 1.0, ds, algorithm="subband")
            _, _, _, prepped = run_prepped(plan, x, 96)
            assert np.array_equal(prepped, O.time_binning(x, 96, ds))


# ------------------------------------------------------------------ multi-range plans
def test_multi_range_plan_matches_reference_calls_per_range():
    """One resident chunk, three (DM range, downsampling) entries as astroflow's
    dmrange list: each range equals the reference GPU path's plain call."""
    from astroflow_b200.dedisp import MultiPlan
    if not O.ref_gpu_available(64):
        pytest.skip("reference GPU build absent")
    spec = ChunkSpec(nchans=512, nsamp=12000, nbits=16, seed=8, rfi_frac=0.08, rfi_amp=6000,
                     impulses=4, imp_amp=5000, pulses=[(300.0, 0.2, 3e-4, 3000.0)])
    x, _ = make_chunk(spec)
    tsamp32, fch1_32, foff32 = float(F32(spec.tsamp)), float(F32(spec.fch1)), float(F32(spec.foff))
    freq = O.freq_table_header(fch1_32, foff32, 512)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    hdr = dict(tsamp=tsamp32, fch1=fch1_32, foff=foff32, nbits=16, nchans=512, ndata=12000)
    iq = IqrmParams(mode=0, radius_frac=0.05, nsigma=3.0, win_sec=0.0, hop_sec=0.0)
    ranges = [(0.0, 100.0, 0.25, 1), (100.0, 400.0, 0.5, 2), (400.0, 1000.0, 1.0, 4)]
    mp = MultiPlan(hdr, ranges, fs, fe, subband_width=64,
                   rfi=RfiParams(use_zero_dm=True, use_iqrm=True, iqrm=iq))
    outs = mp.run(dev(x))
    for (lo, hi, step, ds), o in zip(ranges, outs):
        ref = O.ref_gpu_dedisperse_spec(x, 512, tsamp32, fch1_32, foff32, lo, hi, fs, fe, step, ds,
                                        sb_width=64, use_zero_dm=True, use_iqrm=True, iq=iq)
        assert np.array_equal(to_np(o), ref), f"range {lo}-{hi}"
    mp.close()


def test_delay_tables_match_reference_on_random_plans():
    """Subband delay and residual tables of 40 seeded random plans (bands, DM
    grids, downsampling, subband widths) against the reference GPU build's own
    tables, entry for entry.  Frequencies whose float fch1 + i*foff the reference
    build fuses into one multiply-add put a few delays on the other side of a
    rounding tie when evaluated with two roundings; this sweep catches that."""
    rng = np.random.default_rng(12)
    checked = 0
    for _ in range(40):
        nchans = int(rng.choice([128, 254, 256, 300, 512, 1000, 4096]))
        N = int(rng.integers(2000, 20000))
        tsamp = float(F32(rng.choice([49.152e-6, 64e-6, 1e-4])))
        fhi, bw = float(rng.uniform(1300, 1500)), float(rng.uniform(100, 500))
        foff = float(F32(bw / nchans))
        fch1 = float(F32(fhi - (nchans - 1) * foff))
        freq = O.freq_table_header(fch1, foff, nchans)
        a, b = sorted(rng.uniform(0, 1, 2))
        b = min(max(b, a + 0.2), 1.0)
        fs = float(F32(freq[0] + a * (freq[-1] - freq[0])))
        fe = float(F32(freq[0] + b * (freq[-1] - freq[0])))
        lo = float(rng.choice([0.0, 3.0, 10.5]))
        hi = lo + float(rng.uniform(50, 1500))
        step = float(rng.choice([0.25, 0.5, 1.0, 2.0]))
        ds, sbw = int(rng.choice([1, 2, 4])), int(rng.choice([16, 32, 64]))
        if not O.ref_gpu_available(sbw):
            continue
        hdr = dict(tsamp=tsamp, fch1=fch1, foff=foff, nbits=8, nchans=nchans, ndata=N)
        try:
            plan = Plan(hdr, lo, hi, fs, fe, step, ds, algorithm="subband", subband_width=sbw)
        except ValueError:  # a plan the reference would refuse as well
            continue
        d1, r2 = plan.tables()
        d1r, r2r, _ = O.ref_gpu_tables(nchans, N, tsamp, fch1, foff, lo, hi, fs, fe, step, ds,
                                       sb_width=sbw)
        np.testing.assert_array_equal(d1, d1r)
        np.testing.assert_array_equal(r2, r2r)
        plan.close()
        checked += 1
    if checked == 0:
        pytest.skip("reference GPU builds absent")


def test_full_call_with_rfi_matches_reference_on_random_chunks(tmp_path):
    """Seeded random chunks through the whole plain call (binning, IQRM window
    masks, zero-DM, mask file, both subband stages) against the reference GPU
    call on the same input: IQRM masks and the raw DM-time sums bit for bit."""
    if not O.ref_gpu_available(32):
        pytest.skip("reference GPU build absent")
    rng = np.random.default_rng(31)
    for it in range(8):
        nchans = int(rng.choice([128, 254, 300, 512]))
        N = int(rng.integers(3000, 9000))
        nbits = int(rng.choice([8, 16]))
        ds = int(rng.choice([1, 2]))
        band = None if it % 2 else (float(rng.uniform(0, 0.2)), float(rng.uniform(0.8, 1.0)))
        iqp = (int(rng.integers(0, 2)), float(rng.uniform(0.02, 0.15)), float(rng.uniform(2.0, 4.0)),
               float(rng.choice([0.0, 0.1])), float(rng.choice([0.0, 0.05])))
        case = (nchans, N, nbits, ds, band, iqp)
        x, hdr, freq, fs, fe, iq = rfi_setup(case, seed=100 + it)
        bad = sorted(int(b) for b in rng.choice(nchans, size=4, replace=False))
        mask_file = str(tmp_path / f"m{it}.txt")
        with open(mask_file, "w") as fh:
            fh.write(" ".join(str(b) for b in bad) + "\n")
        hi = float(rng.uniform(100, 400))
        ref_out = O.ref_gpu_dedisperse_spec(x, nchans, hdr["tsamp"], hdr["fch1"], hdr["foff"], 0.0,
                                            hi, fs, fe, 1.0, ds, mask_file=mask_file,
                                            use_mask=True, use_zero_dm=True, use_iqrm=True, iq=iq)
        ref_x, t0, t1, ref_masks = O.ref_gpu_rfi(x, nchans, hdr["tsamp"], hdr["fch1"], hdr["foff"],
                                                 fs, fe, ds, mask_file=mask_file, use_mask=True,
                                                 use_zero_dm=True, use_iqrm=True, iq=iq)
        plan = Plan(hdr, 0.0, hi, fs, fe, 1.0, ds, algorithm="subband",
                    rfi=RfiParams(use_mask=True, use_zero_dm=True, use_iqrm=True, iqrm=iq),
                    bad_channels=bad)
        out, masks, bounds, prepped = run_prepped(plan, x, nchans)
        np.testing.assert_array_equal(masks, ref_masks, err_msg=f"chunk {it}: IQRM masks")
        np.testing.assert_array_equal(prepped, ref_x, err_msg=f"chunk {it}: RFI-processed input")
        np.testing.assert_array_equal(out, ref_out, err_msg=f"chunk {it}: DM-time sums")
