"""The serving loop (astroflow_b200.serve): beams and files submitted together,
overlapping on the device, give the same results as each request alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import IqrmParams, Plan, RfiParams, Stream  # noqa: E402
from astroflow_b200.serve import Server  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


def header_of(spec):
    h = spec.header()
    for k in ("tsamp", "fch1", "foff"):
        h[k] = float(F32(h[k]))
    lo = float(F32(h["fch1"]))
    hi = float(F32(F32(h["fch1"]) + F32(spec.nchans - 1) * F32(h["foff"])))
    return h, lo, hi


def pinned(x):
    t = torch.from_numpy(x.view(np.int16) if x.dtype == np.uint16 else x).pin_memory()
    return t.view(torch.uint16) if x.dtype == np.uint16 else t


def to_dev(x):
    t = torch.from_numpy(x.view(np.int16) if x.dtype == np.uint16 else x).cuda()
    return t.view(torch.uint16) if x.dtype == np.uint16 else t


def test_requests_in_the_mix_equal_requests_alone():
    rfi = RfiParams(use_zero_dm=True, use_iqrm=True,
                    iqrm=IqrmParams(mode=0, radius_frac=0.05, nsigma=3.0, win_sec=0.0, hop_sec=0.0))
    beams = []
    for i, (nch, bits) in enumerate([(256, 8), (128, 16), (256, 8)]):
        spec = ChunkSpec(nchans=nch, nsamp=2000 * 5, nbits=bits, tsamp=64e-6, seed=20 + i,
                         pulses=[(100.0, 0.3, 2e-4, 40.0 if bits == 8 else 4000.0)])
        x, _ = make_chunk(spec)
        h, lo, hi = header_of(spec)
        beams.append((f"b{i}", x, dict(h, ndata=2000), lo, hi))
    files = []
    for i, (nch, n) in enumerate([(512, 9000), (256, 15000)]):
        spec = ChunkSpec(nchans=nch, nsamp=n, nbits=8, tsamp=64e-6, seed=40 + i,
                         pulses=[(200.0, 0.2, 2e-4, 40.0)])
        x, _ = make_chunk(spec)
        h, lo, hi = header_of(spec)
        files.append((x, h, dict(dm_low=0.0, dm_high=300.0, freq_start=lo, freq_end=hi,
                                 dm_step=1.0, subband_width=32, rfi=rfi)))
    srv = Server(hbm_budget_gb=40.0, keep_file_results=True)
    handles = [srv.open_beam(name, h, 0.0, 250.0, lo, hi, 1.0, rfi=rfi) for name, x, h, lo, hi in beams]
    tickets = {name: [] for name, *_ in beams}
    ftickets = []
    chunks = [[pinned(np.ascontiguousarray(x[k * 2000:(k + 1) * 2000])) for k in range(5)]
              for _, x, *_ in beams]
    got = {name: [] for name, *_ in beams}
    for k in range(5):
        for (name, *_), b, cs in zip(beams, handles, chunks):
            tickets[name].append(srv.submit_chunk(b, cs[k]))
        if k < len(files):
            x, h, kw = files[k]
            ftickets.append(srv.submit_file(pinned(x), h, kw))
        # step until this round's chunks are done, copying results before the ring reuses them
        while any(t.done is None for ts in tickets.values() for t in ts):
            srv.step()
        for name in tickets:
            got[name].append(tickets[name][-1].result.copy())
    srv.drain()
    st = srv.stats()
    assert not st["errors"] and st["chunks"]["n"] == 15 and st["files"]["n"] == 2
    for (name, x, h, lo, hi) in beams:
        alone = Stream(h, 0.0, 250.0, lo, hi, 1.0, rfi=rfi)
        for k in range(5):
            want = alone.push(to_dev(np.ascontiguousarray(x[k * 2000:(k + 1) * 2000])))
            want = want.view(torch.int32).cpu().numpy().view(np.uint32)
            assert np.array_equal(got[name][k], want), f"{name} chunk {k}"
        alone.close()
    for t, (x, h, kw) in zip(ftickets, files):
        plan = Plan(h, **kw)
        want = plan.run(to_dev(x)).view(torch.int32).cpu().numpy()
        assert np.array_equal(t.result.view(torch.int32).cpu().numpy(), want)
        assert t.latency is not None and t.latency > 0
    srv.close()
