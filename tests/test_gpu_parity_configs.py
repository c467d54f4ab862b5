"""Parity at the benchmarked configurations, across time tiles, against the
reference's own code run on the same inputs.

  * the wideband subband configuration (4096 channels of 8-bit samples, DM
    0-3000 in steps of 0.5, subband width 64, IQRM with radius 5 lags at 3
    sigma, zero-DM as called, sinusoidal RFI channels, broadband impulses and
    three pulses) on 2^18 samples, six time tiles of the library's subband-sum
    pipeline, against the reference GPU build (src/core/dedispered.cu:1124-1235
    tiles the same chunk its own way): every DM row and column, and the IQRM
    masks;
  * the brute-force configuration at its full size (1024 channels, 2^17
    samples, 1001 DMs) against the reference's CPU path
    (include/cpucal.hpp:75-201) with the library's default delay table (no
    table injected);
  * two of the three DM ranges of the 8192-channel 16-bit configuration (width
    64, 128 subbands; IQRM, zero-DM, 8% RFI channels) on 2^18 samples, four and
    two time tiles;
  * six chunks of the heterogeneous batch draw, run as grouped and persistent
    batches, each against the reference GPU call on that chunk;
  * the range zero-DM filter in the reference's arithmetic (DD_ZDM_RANGE_REF)
    against the reference's own range kernels (src/rfi/rfimarker.cu:172-305),
    on 8- and 16-bit samples over 4096 channels, where 16-bit float sums pass 2^24.
Integer outputs and masks are compared bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import Batch, IqrmParams, Plan, RfiParams  # noqa: E402
from astroflow_b200.synth import ChunkSpec, draw_batch, make_chunk, make_chunk_device  # noqa: E402

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
    return torch.from_numpy(x).cuda()


def header32(spec):
    """The Header the reference's _dedisperse_spec path receives (float fields)."""
    hdr = dict(tsamp=float(F32(spec.tsamp)), fch1=float(F32(spec.fch1)),
               foff=float(F32(spec.foff)), nbits=spec.nbits, nchans=spec.nchans,
               ndata=spec.nsamp)
    freq = O.freq_table_header(hdr["fch1"], hdr["foff"], spec.nchans)
    return hdr, float(F32(freq[0])), float(F32(freq[-1]))


def assert_rows_equal(out, ref, block=256):
    """Device output against the reference's host array, a block of rows at a time."""
    assert tuple(out.shape) == ref.shape
    for r0 in range(0, ref.shape[0], block):
        got = to_np(out[r0:r0 + block])
        want = ref[r0:r0 + block]
        if not np.array_equal(got, want):
            bad = np.argwhere(got != want)
            r, c = bad[0]
            raise AssertionError(f"{len(bad)} samples differ in rows {r0}-{r0 + block}; first "
                                 f"at row {r0 + r}, column {c}: {got[r, c]} != {want[r, c]}")


WIDE_IQ = IqrmParams(mode=1, radius_frac=0.00134, nsigma=3.0, geofactor=1.5, win_sec=0.0,
                     hop_sec=0.5, include_tail=True)


def test_wideband_4096ch_2e18_across_six_tiles_matches_reference_gpu():
    if not O.ref_gpu_available(64):
        pytest.skip("reference GPU build absent")
    spec = ChunkSpec(nchans=4096, nsamp=1 << 18, nbits=8, seed=1234, rfi_frac=0.05, rfi_amp=60.0,
                     impulses=20, imp_amp=50.0,
                     pulses=[(120.0, 1.0, 1e-3, 12.0), (780.0, 4.0, 1e-3, 12.0),
                             (2400.0, 2.0, 1e-3, 12.0)])
    xd, _ = make_chunk_device(spec, 0)
    x = xd.cpu().numpy()
    hdr, fs, fe = header32(spec)
    rfi = RfiParams(use_zero_dm=True, use_iqrm=True, iqrm=WIDE_IQ)
    plan = Plan(hdr, 0.0, 3000.0, fs, fe, 0.5, 1, algorithm="subband", subband_width=64, rfi=rfi)
    info = plan.info
    assert (info["dm_steps"], info["nsb"]) == (6001, 64)
    ntiles = -(-info["out_cols"] // info["tile_samples"])
    assert ntiles >= 3, f"{ntiles} time tiles"
    masks = torch.zeros((1, 4096), dtype=torch.uint8, device="cuda")
    bounds = torch.zeros((1, 2), dtype=torch.int32, device="cuda")
    out = plan.run(xd, iqrm_masks=masks, iqrm_bounds=bounds)
    torch.cuda.synchronize()
    _, t0, t1, ref_masks = O.ref_gpu_rfi(x, 4096, hdr["tsamp"], hdr["fch1"], hdr["foff"], fs, fe, 1,
                                         use_zero_dm=True, use_iqrm=True, iq=WIDE_IQ, sb_width=64)
    assert np.array_equal(masks.cpu().numpy(), ref_masks)
    assert int(ref_masks.sum()) > 0
    ref = O.ref_gpu_dedisperse_spec_rows(x, 4096, hdr["tsamp"], hdr["fch1"], hdr["foff"], 0.0,
                                         3000.0, fs, fe, 0.5, 1, sb_width=64, use_zero_dm=True,
                                         use_iqrm=True, iq=WIDE_IQ)
    assert_rows_equal(out, ref)
    plan.close()


def test_brute_1024ch_2e17_1001dm_matches_reference_cpu_with_default_table():
    if not O.ref_cpu_available():
        pytest.skip("reference CPU build absent")
    spec = ChunkSpec(nchans=1024, nsamp=1 << 17, nbits=8, seed=0,
                     pulses=[(565.0, 2.0, 1e-3, 12.0)])
    x, _ = make_chunk(spec)
    hdr = dict(tsamp=float(F32(spec.tsamp)), fch1=float(F32(spec.fch1)),
               foff=float(F32(spec.foff)), nbits=8, nchans=1024, ndata=spec.nsamp)
    freq = O.freq_table_fil(hdr["fch1"], hdr["foff"], 1024)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    t_sample = float(F32(spec.nsamp * hdr["tsamp"] * 0.999))
    plan = Plan(hdr, 0.0, 1000.0, fs, fe, 1.0, 1, t_sample, algorithm="brute", freq_mode="fil")
    assert plan.out_shape[0] == 1001
    out = to_np(plan.run(dev(x)))
    ref = np.concatenate(O.ref_bruteforce_cpu(x, 1024, hdr["fch1"], hdr["foff"], hdr["tsamp"], 0.0,
                                              1000.0, fs, fe, 1.0, 1, t_sample), axis=1)
    assert out.shape == ref.shape
    assert np.array_equal(out, ref), f"{int((out != ref).sum())} samples differ"
    plan.close()


LARGE_IQ = IqrmParams(mode=1, radius_frac=0.00067, nsigma=3.0, geofactor=1.5, win_sec=0.0,
                      hop_sec=0.5, include_tail=True)


@pytest.mark.parametrize("lo,hi,step,ds,min_tiles", [(0.0, 500.0, 0.25, 1, 3),
                                                      (2000.0, 5000.0, 1.0, 4, 2)])
def test_large_8192ch_u16_range_matches_reference_gpu(lo, hi, step, ds, min_tiles):
    if not O.ref_gpu_available(64):
        pytest.skip("reference GPU build absent")
    spec = ChunkSpec(nchans=8192, nsamp=1 << 18, nbits=16, seed=4321, rfi_frac=0.08,
                     rfi_amp=6000.0, impulses=20, imp_amp=5000.0,
                     pulses=[(300.0, 2.0, 1e-3, 1200.0), (3500.0, 6.0, 1e-3, 1200.0)])
    xd, _ = make_chunk_device(spec, 0)
    x = xd.view(torch.int16).cpu().numpy().view(np.uint16)
    hdr, fs, fe = header32(spec)
    rfi = RfiParams(use_zero_dm=True, use_iqrm=True, iqrm=LARGE_IQ)
    plan = Plan(hdr, lo, hi, fs, fe, step, ds, algorithm="subband", subband_width=64, rfi=rfi)
    assert plan.info["nsb"] == 128
    ntiles = -(-plan.info["out_cols"] // plan.info["tile_samples"])
    assert ntiles >= min_tiles, f"{ntiles} time tiles"
    out = plan.run(xd)
    ref = O.ref_gpu_dedisperse_spec_rows(x, 8192, hdr["tsamp"], hdr["fch1"], hdr["foff"], lo, hi,
                                         fs, fe, step, ds, sb_width=64, use_zero_dm=True,
                                         use_iqrm=True, iq=LARGE_IQ)
    assert_rows_equal(out, ref)
    plan.close()


BATCH_PICK = [0, 1, 3, 4, 8, 13]  # 8/16-bit, 1024-4096 channels, both bands, ds 1-8


@pytest.mark.parametrize("persistent", [False, True])
def test_batch_draw_chunks_match_reference_gpu(persistent):
    if not O.ref_gpu_available(32):
        pytest.skip("reference GPU build absent")
    chunks = [draw_batch(64, seed=2024, subband_width=32)[i] for i in BATCH_PICK]
    plans, xs, outs, hosts = [], [], [], []
    for c in chunks:
        hdr, fs, fe = header32(c.spec)
        plans.append(Plan(hdr, 0.0, c.dm_high, fs, fe, c.dm_step, c.time_downsample,
                          algorithm="subband", subband_width=32))
        xd, _ = make_chunk_device(c.spec, 0)
        xs.append(xd)
        outs.append(plans[-1].empty_output())
        hosts.append((xd if c.spec.nbits == 8 else xd.view(torch.int16)).cpu().numpy())
    batch = Batch(plans, use_graph=True, persistent=persistent)
    batch.run(xs, outs)
    batch.status()
    for c, p, o, h in zip(chunks, plans, outs, hosts):
        if c.spec.nbits == 16:
            h = h.view(np.uint16)
        hdr, fs, fe = header32(c.spec)
        ref = O.ref_gpu_dedisperse_spec_rows(h, c.spec.nchans, hdr["tsamp"], hdr["fch1"],
                                             hdr["foff"], 0.0, c.dm_high, fs, fe, c.dm_step,
                                             c.time_downsample, sb_width=32)
        assert_rows_equal(o, ref)
    batch.close()
    for p in plans:
        p.close()


@pytest.mark.parametrize("nbits,band,iqrm", [(8, (0.0, 1.0), False), (16, (0.0, 1.0), False),
                                              (16, (0.0, 1.0), True), (16, (0.1, 0.9), False)])
def test_zero_dm_range_ref_matches_reference_range_kernels(nbits, band, iqrm):
    if not O.ref_gpu_available(32):
        pytest.skip("reference GPU build absent")
    spec = ChunkSpec(nchans=4096, nsamp=3000, nbits=nbits, seed=77, rfi_frac=0.05,
                     rfi_amp=60 if nbits == 8 else 6000, impulses=8,
                     imp_amp=50 if nbits == 8 else 5000)
    x, _ = make_chunk(spec)
    hdr, f0, f1 = header32(spec)
    fs = float(F32(f0 + band[0] * (f1 - f0)))
    fe = float(F32(f0 + band[1] * (f1 - f0)))
    iq = IqrmParams(mode=1, radius_frac=0.002, nsigma=3.0, win_sec=0.0, hop_sec=0.0)
    rfi = RfiParams(use_zero_dm=True, use_iqrm=iqrm, iqrm=iq)
    outs = {}
    for mode in ("range_ref", "range"):
        plan = Plan(hdr, 0.0, 50.0, fs, fe, 1.0, 1, algorithm="subband", zero_dm_mode=mode, rfi=rfi)
        prepped = torch.zeros((spec.nsamp, 4096), dtype=dev(x[:1]).dtype, device="cuda")
        nw = max(int(plan.info["n_iqrm_windows"]), 1)
        plan.run(dev(x), iqrm_masks=torch.zeros((nw, 4096), dtype=torch.uint8, device="cuda"),
                 prepped=prepped)
        outs[mode] = to_np(prepped)
        cs, ce = int(plan.info["chan_start"]), int(plan.info["chan_end"])
        plan.close()
    src = x
    if iqrm:  # the reference's IQRM window masks first, as its call site orders them
        src, _, _, _ = O.ref_gpu_rfi(x, 4096, hdr["tsamp"], hdr["fch1"], hdr["foff"], fs, fe, 1,
                                     use_iqrm=True, iq=iq)
    ref = O.ref_gpu_zero_dm_range(src, 4096, cs, ce)
    assert not np.array_equal(ref, src)  # the filter changed something
    assert np.array_equal(outs["range_ref"], ref), \
        f"{int((outs['range_ref'] != ref).sum())} samples differ"
