"""The autotuner of the subband path (dd_plan_autotune): it only reschedules the
same sums, so a tuned plan's DM-time output equals the untuned plan's bit for
bit, and both equal the oracle's sums with the plan's tables."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import Plan  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


def _dev(x):
    v = {np.uint8: (x, torch.uint8), np.uint16: (x.view(np.int16), torch.uint16)}[x.dtype.type]
    return torch.from_numpy(v[0].reshape(-1)).cuda().view(v[1])


def _host(t):
    return t.view(torch.int32).cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("nchans,n,nbits,sbw", [(512, 60000, 8, 64), (256, 40000, 16, 32)])
def test_tuned_plan_gives_the_same_sums(nchans, n, nbits, sbw):
    spec = ChunkSpec(nchans=nchans, nsamp=n, nbits=nbits, seed=5,
                     pulses=[(150.0, 0.2 * n * 49.152e-6, 2e-4, 30.0 if nbits == 8 else 3000.0)])
    x, _ = make_chunk(spec)
    hdr = spec.header()
    hdr.update(tsamp=float(F32(hdr["tsamp"])), fch1=float(F32(hdr["fch1"])), foff=float(F32(hdr["foff"])))
    fs = hdr["fch1"]
    fe = float(F32(F32(hdr["fch1"]) + F32(nchans - 1) * F32(hdr["foff"])))
    plan = Plan(hdr, 0.0, 400.0, fs, fe, 0.5, 1, algorithm="subband", subband_width=sbw)
    xd = _dev(x)
    before = _host(plan.run(xd))
    rep = plan.autotune(xd, reps=1)
    assert rep["candidates"] >= 2 and rep["best_ms"] <= rep["default_ms"] + 1e-9
    assert rep["best_stages"] in (0, 4, 6, 8) and rep["best_tile_samples"] > 0
    assert plan.info["tile_samples"] == rep["best_tile_samples"]
    after = _host(plan.run(xd))
    np.testing.assert_array_equal(after, before)
    d1, r2 = plan.tables()
    freq = O.freq_table_header(hdr["fch1"], hdr["foff"], nchans)
    op = O.subband_plan(freq, n, 0.0, 400.0, fs, fe, 0.5, 1, sb_width=sbw)
    np.testing.assert_array_equal(after, O.subband_sums(x, nchans, op, d1, r2).astype(np.uint32))
    plan.close()


def test_autotune_refuses_the_brute_force_path():
    hdr = dict(tsamp=64e-6, fch1=1200.0, foff=1.0, nbits=8, nchans=64, ndata=4096)
    plan = Plan(hdr, 0.0, 50.0, 1200.0, 1263.0, 1.0, 1, 0.1, algorithm="brute")
    x = torch.zeros(4096 * 64, dtype=torch.uint8, device="cuda")
    with pytest.raises(RuntimeError):
        plan.autotune(x)
    plan.close()
