"""The allocation-free IQRM entry point (dd_iqrm_masks_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory while they run
(deadline-bound real-time loops, frameworks that own the GPU's memory); its
working memory is a static per-GPU array.  Its masks must equal the plan path's
(dd_run_ex) bit for bit, on two calls in a row, so that nothing a call leaves in
the shared array changes the next call.  Cases: 8-, 16- and 32-bit samples, the
full band and a channel sub-range (chan_start > 0), one window and many, and a
one-channel band, where IQRM has no lags and every mask is zero.  This file is
collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import IqrmParams, Plan, RfiParams, iqrm_masks_noalloc  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


def to_dev(x):
    if x.dtype == np.uint16:
        return torch.from_numpy(x.view(np.int16)).cuda().view(torch.uint16)
    if x.dtype == np.uint32:
        return torch.from_numpy(x.view(np.int32)).cuda().view(torch.uint32)
    return torch.from_numpy(x).cuda()


def chunk(nbits, nchans, nsamp=6000, seed=5):
    amp = {8: (60, 50), 16: (6000, 5000), 32: (6e5, 5e5)}[nbits]
    spec = ChunkSpec(nchans=nchans, nsamp=nsamp, nbits=nbits, seed=seed, rfi_frac=0.06,
                     impulses=5, rfi_amp=amp[0], imp_amp=amp[1])
    x, _ = make_chunk(spec)
    hdr = dict(tsamp=float(F32(spec.tsamp)), fch1=float(F32(spec.fch1)),
               foff=float(F32(spec.foff)), nbits=nbits, nchans=nchans, ndata=spec.nsamp)
    return x, hdr


def compare_twice(x, hdr, iq, band=(0.0, 1.0), expect_flags=True):
    """Plan-path masks (dd_run_ex) against two no-alloc calls in a row."""
    nchans = hdr["nchans"]
    freq = F32(hdr["fch1"]) + np.arange(nchans, dtype=F32) * F32(hdr["foff"])
    fs = float(F32(freq[0] + band[0] * (freq[-1] - freq[0])))
    fe = float(F32(freq[0] + band[1] * (freq[-1] - freq[0])))
    plan = Plan(hdr, 0.0, 50.0, fs, fe, 1.0, 1, algorithm="subband",
                rfi=RfiParams(use_iqrm=True, iqrm=iq))
    nwin = int(plan.info["n_iqrm_windows"])
    xd = to_dev(x)
    ref_masks = torch.zeros((nwin, nchans), dtype=torch.uint8, device="cuda")
    ref_bounds = torch.zeros((nwin, 2), dtype=torch.int32, device="cuda")
    plan.run(xd, iqrm_masks=ref_masks, iqrm_bounds=ref_bounds)
    cs, ce = int(plan.info["chan_start"]), int(plan.info["chan_end"])
    tsamp_iqrm = float(F32(hdr["tsamp"]))  # no downsampling: the IQRM stage's sampling time
    for _ in range(2):
        masks = torch.full((nwin + 2, nchans), 7, dtype=torch.uint8, device="cuda")
        bounds = torch.zeros((nwin + 2, 2), dtype=torch.int32, device="cuda")
        n = iqrm_masks_noalloc(xd, nchans, cs, ce, tsamp_iqrm, iq, masks, bounds)
        torch.cuda.synchronize()
        assert n == nwin
        assert torch.equal(masks[:n], ref_masks)
        assert torch.equal(bounds[:n], ref_bounds)
    assert (int(ref_masks.sum()) > 0) == expect_flags
    plan.close()
    return cs, nwin


@pytest.mark.parametrize("nbits,nchans,win_sec,mode,band", [
    (8, 512, 0.0, 1, (0.0, 1.0)),
    (16, 384, 0.1, 0, (0.0, 1.0)),
    (32, 256, 0.05, 1, (0.0, 1.0)),
    (8, 300, 0.05, 0, (0.2, 0.9)),
])
def test_noalloc_masks_equal_plan_path_twice(nbits, nchans, win_sec, mode, band):
    x, hdr = chunk(nbits, nchans)
    iq = IqrmParams(mode=mode, radius_frac=0.1, nsigma=3.0, geofactor=1.5, win_sec=win_sec,
                    hop_sec=0.05, include_tail=True)
    cs, nwin = compare_twice(x, hdr, iq, band)
    assert (cs > 0) == (band[0] > 0)
    assert (nwin > 1) == (win_sec > 0)


def test_noalloc_one_channel_band_has_no_lags():
    """Two channels, so the IQRM band [chan_start, chan_end) holds one channel:
    no lag fits, and both paths leave every mask at zero."""
    rng = np.random.default_rng(9)
    x = rng.integers(0, 256, size=(4000, 2)).astype(np.uint8)
    hdr = dict(tsamp=float(F32(64e-6)), fch1=1400.0, foff=1.0, nbits=8, nchans=2, ndata=4000)
    iq = IqrmParams(mode=0, radius_frac=0.5, nsigma=3.0, win_sec=0.0, hop_sec=0.0)
    compare_twice(x, hdr, iq, expect_flags=False)


def test_noalloc_rejects_too_few_windows():
    x, hdr = chunk(8, 128)
    xd = to_dev(x)
    iq = IqrmParams(mode=0, radius_frac=0.1, nsigma=3.0, win_sec=0.05, hop_sec=0.05)
    masks = torch.zeros((8, 128), dtype=torch.uint8, device="cuda")
    bounds = torch.zeros((8, 2), dtype=torch.int32, device="cuda")
    n = iqrm_masks_noalloc(xd, 128, 0, 127, float(F32(hdr["tsamp"])), iq, masks, bounds)
    assert n > 1
    with pytest.raises(ValueError, match="max_windows"):
        iqrm_masks_noalloc(xd, 128, 0, 127, float(F32(hdr["tsamp"])), iq, masks[: n - 1],
                           bounds[: n - 1])


def test_noalloc_rejects_oversized_request():
    nchans = 16384
    x = torch.zeros((64, nchans), dtype=torch.uint8, device="cuda")
    iq = IqrmParams(mode=0, radius_frac=0.5, nsigma=3.0, win_sec=1e-4, hop_sec=1e-5)
    masks = torch.zeros((64, nchans), dtype=torch.uint8, device="cuda")
    bounds = torch.zeros((64, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError, match="static scratch"):
        iqrm_masks_noalloc(x, nchans, 0, nchans - 1, 1e-5, iq, masks, bounds)


def test_noalloc_rejects_band_wider_than_the_sort():
    """A band whose per-window sort buffer exceeds the block's shared memory is
    refused with a message giving the limit, before anything is launched."""
    nchans = 100000
    x = torch.zeros((8, nchans), dtype=torch.uint8, device="cuda")
    iq = IqrmParams(mode=0, radius_frac=1e-5, nsigma=3.0, win_sec=0.0, hop_sec=0.0)
    masks = torch.zeros((1, nchans), dtype=torch.uint8, device="cuda")
    bounds = torch.zeros((1, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError, match="shared memory"):
        iqrm_masks_noalloc(x, nchans, 0, nchans - 1, 1e-3, iq, masks, bounds)
