"""The oracle against the reference's own CPU build, the golden fixtures and
known-answer cases (no GPU needed)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

F32 = np.float32
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_known_answer_dm0_is_channel_sum():
    """DM 0: every channel delay is 0, so each output sample is the sum of the
    band's channels at that sample (the identity the reference's own test uses,
    python/tests/test_dedispered.py:21-62); the CPU path leaves out the top channel."""
    rng = np.random.default_rng(0)
    x = rng.integers(0, 256, size=(700, 40)).astype(np.uint8)
    freq = O.freq_table_fil(1200.0, 1.0, 40)
    out = O.bruteforce_cpu(x, 40, freq, 1e-3, 0.0, 0.0, float(F32(freq[0])), float(F32(freq[-1])),
                           1.0, 1, 0.7)
    assert len(out) == 1 and out[0].shape == (1, 700)
    assert np.array_equal(out[0][0], x[:, :39].sum(axis=1))


def test_known_answer_single_channel_impulse():
    """An impulse in channel c at sample T lands at column T - delay[m][c] of every DM row."""
    nchans, N = 32, 3000
    freq = O.freq_table_fil(1100.0, 2.0, nchans)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    cs, ce = O.chan_range(freq, fs, fe)
    d = O.cpu_delay_table(freq, cs, ce, 0.0, 5.0, 21, 1e-4)
    for c in (0, 7, 30):
        x = np.zeros((N, nchans), np.uint8)
        x[N - 1, c] = 9
        out = np.concatenate(O.bruteforce_cpu(x, nchans, freq, 1e-4, 0.0, 100.0, fs, fe, 5.0, 1, N * 1e-4 * 0.999), axis=1)
        for m in range(21):
            nz = np.nonzero(out[m])[0]
            assert list(nz) == [N - 1 - d[m][c]] and out[m][nz[0]] == 9


def test_known_answer_constant_input_subband():
    """Constant input c: away from the end of the chunk every output equals c times
    the number of channels in the band, whatever the delay tables are."""
    nchans, N, c = 96, 4000, 3
    x = np.full((N, nchans), c, np.uint8)
    freq = O.freq_table_header(1000.0, 5.0, nchans)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    plan = O.subband_plan(freq, N, 0.0, 30.0, fs, fe, 0.2, 1, sb_width=32)
    d1, r2 = O.subband_tables_ieee(freq, plan, 0.0, 0.2, 1e-4, 1)
    out = O.subband_sums(x, nchans, plan, d1, r2)
    edge = int(d1.max() + r2.max())
    assert edge < N // 2
    assert np.all(out[:, : N - edge - 1] == c * nchans)
    # past that point terms drop out (t + delay >= N contributes nothing)
    assert out[-1, N - 1] < c * nchans


def test_iqrm_flags_an_outlier_channel():
    rng = np.random.default_rng(1)
    x = np.clip(np.rint(rng.normal(128, 20, size=(4000, 128))), 0, 255).astype(np.uint8)
    x[:, 40] = np.clip(x[:, 40].astype(int) + 60, 0, 255).astype(np.uint8)
    m = O.iqrm_window_mask(x, 128, 0, 4000, 0, 127, 0, 0.1, 3.0, 1.5)
    assert m[40] == 1 and m.sum() <= 4


def test_zero_dm_callsite_is_noop_at_chan_start_zero():
    rng = np.random.default_rng(2)
    x = rng.integers(0, 256, size=(500, 64)).astype(np.uint8)
    y = x.copy()
    O.zero_dm_callsite(y, 0, 63, 500)
    assert np.array_equal(x, y)


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
def test_oracle_pinned_to_reference_cpu_build():
    """Random configurations (8/16-bit, downsampling, slicing, sub-bands): with the
    reference build's delay table injected the oracle's sums are identical, and the
    IEEE table the oracle and the GPU library use differs from the reference build's
    only at a small fraction of rounding ties."""
    rng = np.random.default_rng(21)
    nbad = ntab = 0
    for _ in range(10):
        nchans = int(rng.integers(8, 160))
        tsamp = float(rng.choice([64e-6, 49.152e-6, 1e-4, 3.2e-5]))
        fch1, foff = float(rng.uniform(800, 1500)), float(rng.uniform(0.1, 2.0))
        lo, step = float(np.round(rng.uniform(0, 20), 2)), float(rng.choice([1.0, 0.5, 0.3, 0.7, 2.3]))
        hi = lo + step * int(rng.integers(10, 50))
        N, ds = int(rng.integers(400, 2500)), int(rng.choice([1, 2, 3]))
        tsl = float(N * tsamp * rng.uniform(0.2, 1.0))
        nbits = int(rng.choice([8, 16]))
        x = rng.integers(0, 256 if nbits == 8 else 65536, size=(N, nchans)).astype(np.uint8 if nbits == 8 else np.uint16)
        freq = O.freq_table_fil(fch1, foff, nchans)
        fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
        D = O.ref_cpu_delays(nchans, N, fch1, foff, tsamp, lo, hi, fs, fe, step)
        cs, ce = O.chan_range(freq, fs, fe)
        nbad += int((O.cpu_delay_table(freq, cs, ce, lo, step, D.shape[0], tsamp) != D).sum())
        ntab += D.size
        ref = O.ref_bruteforce_cpu(x, nchans, fch1, foff, tsamp, lo, hi, fs, fe, step, ds, tsl)
        orc = O.bruteforce_cpu(x, nchans, freq, tsamp, lo, hi, fs, fe, step, ds, tsl, delay=D)
        assert len(orc) == len(ref)
        for a, b in zip(orc, ref):
            assert a.shape == b.shape and np.array_equal(a, b)
    assert nbad <= max(3, ntab // 1000)


def golden_files(prefix):
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(os.path.join(GOLDEN, f) for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))


@pytest.mark.parametrize("path", golden_files("ref_cpu_"), ids=os.path.basename)
def test_oracle_matches_reference_cpu_golden(path):
    """Fixtures produced by the reference's cpucal::dedispered_fil_omp (see
    tests/golden/make_golden.py); the oracle reproduces the stored sums from the
    stored reference delay table."""
    g = np.load(path)
    x = g["data"]
    nchans = int(g["nchans"])
    freq = O.freq_table_fil(float(g["fch1"]), float(g["foff"]), nchans)
    kw = dict(tsamp=float(g["tsamp"]), dm_low=float(g["dm_low"]), dm_high=float(g["dm_high"]),
              freq_start=float(g["freq_start"]), freq_end=float(g["freq_end"]),
              dm_step=float(g["dm_step"]), ds=int(g["ds"]), t_sample=float(g["t_sample"]))
    out = O.bruteforce_cpu(x, nchans, freq, kw["tsamp"], kw["dm_low"], kw["dm_high"], kw["freq_start"],
                           kw["freq_end"], kw["dm_step"], kw["ds"], kw["t_sample"], delay=g["delay"])
    assert np.array_equal(np.concatenate(out, axis=1), g["out"])
    cs, ce = O.chan_range(freq, kw["freq_start"], kw["freq_end"])
    ieee = O.cpu_delay_table(freq, cs, ce, kw["dm_low"], kw["dm_step"], g["delay"].shape[0], kw["tsamp"])
    assert int((ieee != g["delay"]).sum()) <= max(2, g["delay"].size // 1000)


@pytest.mark.parametrize("path", golden_files("ref_gpu_sub_"), ids=os.path.basename)
def test_oracle_subband_sums_match_reference_gpu_golden(path):
    """Fixtures produced by the reference's gpucal::dedisperse_spec on a B200 (see
    tests/golden/make_golden.py): the oracle's channel range, DM count and subband
    sums (from the stored reference tables) reproduce the stored raw output."""
    g = np.load(path)
    x, nchans, ds = g["data"], int(g["nchans"]), int(g["ds"])
    freq = O.freq_table_header(float(g["fch1"]), float(g["foff"]), nchans)
    plan = O.subband_plan(freq, x.shape[0], float(g["dm_low"]), float(g["dm_high"]),
                          float(g["freq_start"]), float(g["freq_end"]), float(g["dm_step"]), ds,
                          sb_width=int(g["sb_width"]))
    assert (plan.chan_start, plan.chan_end) == (int(g["chan_start"]), int(g["chan_end"]))
    assert plan.dm_steps == g["out"].shape[0]
    xb = O.time_binning(x, nchans, ds) if ds > 1 else x
    out = O.subband_sums(xb, nchans, plan, g["delay1"], g["residual2"])
    assert np.array_equal(out, g["out"].astype(np.uint64))


@pytest.mark.parametrize("path", golden_files("ref_gpu_rfi_"), ids=os.path.basename)
def test_oracle_rfi_stages_match_reference_gpu_golden(path):
    """The RFI stages of the reference GPU call (binning, IQRM window masks, zero-DM
    at the reference's call site, mask file) from the fixtures: the oracle gives the
    same window bounds, masks and processed input."""
    import types

    g = np.load(path)
    x, nchans, ds = g["data"], int(g["nchans"]), int(g["ds"])
    freq = O.freq_table_header(float(g["fch1"]), float(g["foff"]), nchans)
    cs, ce = O.chan_range(freq, float(g["freq_start"]), float(g["freq_end"]))
    mode, rf, ns, win, hop = (float(v) for v in g["iq"])
    iq = types.SimpleNamespace(mode=int(mode), radius_frac=rf, nsigma=ns, geofactor=1.5,
                               win_sec=win, hop_sec=hop, include_tail=True)
    xb = O.time_binning(x, nchans, ds) if ds > 1 else x.copy()
    t0, t1, masks = O.iqrm_masks(xb, nchans, cs, ce, float(F32(F32(g["tsamp"]) * F32(ds))), iq)
    assert np.array_equal(t0, g["win_t0"]) and np.array_equal(t1, g["win_t1"])
    assert np.array_equal(masks, g["masks"])
    O.apply_window_masks(xb, nchans, t0, t1, masks)
    if bool(g["use_zero_dm"]):
        O.zero_dm_callsite(xb, cs, ce, xb.shape[0])
    if bool(g["use_mask"]):
        O.mark_channels(xb, nchans, [int(c) for c in g["bad"]])
    assert np.array_equal(xb, g["processed"])
