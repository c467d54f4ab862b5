"""The allocation-free IQRM entry point (dd_iqrm_masks_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory while they run
(deadline-bound real-time loops, frameworks that own the GPU's memory); its
working memory is a static per-GPU array.  Its masks must equal the plan path's
(dd_run_ex) bit for bit, on two calls in a row, so that nothing a call leaves in
the shared array changes the next call.  This file is collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import IqrmParams, Plan, RfiParams, iqrm_masks_noalloc  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


@pytest.mark.parametrize("nbits,nchans,win_sec,mode", [(8, 512, 0.0, 1), (16, 384, 0.1, 0)])
def test_noalloc_masks_equal_plan_path_twice(nbits, nchans, win_sec, mode):
    spec = ChunkSpec(nchans=nchans, nsamp=6000, nbits=nbits, seed=5, rfi_frac=0.06, impulses=5,
                     rfi_amp=60 if nbits == 8 else 6000, imp_amp=50 if nbits == 8 else 5000)
    x, _ = make_chunk(spec)
    hdr = dict(tsamp=float(F32(spec.tsamp)), fch1=float(F32(spec.fch1)), foff=float(F32(spec.foff)),
               nbits=nbits, nchans=nchans, ndata=spec.nsamp)
    freq = F32(hdr["fch1"]) + np.arange(nchans, dtype=F32) * F32(hdr["foff"])
    fs, fe = float(freq[0]), float(freq[-1])
    iq = IqrmParams(mode=mode, radius_frac=0.1, nsigma=3.0, geofactor=1.5, win_sec=win_sec,
                    hop_sec=0.05, include_tail=True)
    plan = Plan(hdr, 0.0, 50.0, fs, fe, 1.0, 1, algorithm="subband",
                rfi=RfiParams(use_iqrm=True, iqrm=iq))
    nwin = int(plan.info["n_iqrm_windows"])
    xd = torch.from_numpy(x.view(np.int16) if nbits == 16 else x).cuda()
    if nbits == 16:
        xd = xd.view(torch.uint16)
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
        assert int(ref_masks.sum()) > 0


def test_noalloc_rejects_oversized_request():
    nchans = 16384
    x = torch.zeros((64, nchans), dtype=torch.uint8, device="cuda")
    iq = IqrmParams(mode=0, radius_frac=0.5, nsigma=3.0, win_sec=1e-4, hop_sec=1e-5)
    masks = torch.zeros((64, nchans), dtype=torch.uint8, device="cuda")
    bounds = torch.zeros((64, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError, match="static scratch"):
        iqrm_masks_noalloc(x, nchans, 0, nchans - 1, 1e-5, iq, masks, bounds)
