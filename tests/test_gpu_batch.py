"""Batched runs (dd_batch_*): many chunks of different geometries in one persistent
launch, with and without CUDA-graph replay, must equal each plan's own run bit for
bit; a new set of buffers is captured anew."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import Batch, IqrmParams, Plan, RfiParams  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


def to_np(t):
    return t.view(torch.int32).cpu().numpy().view(np.uint32)


def dev(x):
    if x.dtype == np.uint16:
        return torch.from_numpy(x.view(np.int16)).cuda().view(torch.uint16)
    return torch.from_numpy(x).cuda()


# nchans, nsamp, nbits, f_hi, bw, dm_high, dm_step, ds, sbw, algorithm, rfi
CHUNKS = [
    (1024, 9000, 8, 1500.0, 500.0, 500.0, 1.0, 1, 32, "subband", True),
    (2048, 6000, 16, 1550.0, 300.0, 300.0, 2.0, 2, 64, "subband", True),
    (512, 12000, 8, 1500.0, 500.0, 1000.0, 0.5, 4, 16, "subband", False),
    (4096, 4096, 8, 1500.0, 500.0, 200.0, 1.0, 1, 64, "subband", False),
    (256, 20000, 16, 1500.0, 500.0, 800.0, 1.5, 8, 32, "subband", True),
    (300, 7000, 8, 1500.0, 400.0, 300.0, 1.0, 1, 32, "brute", False),
    (1000, 5000, 8, 1500.0, 500.0, 1500.0, 2.0, 2, 300, "subband", False),
]


def make(case, seed):
    nchans, n, nbits, f_hi, bw, dmh, step, ds, sbw, algo, rfi = case
    spec = ChunkSpec(nchans=nchans, nsamp=n, nbits=nbits, f_hi=f_hi, bandwidth=bw,
                     tsamp=64e-6, seed=seed, rfi_frac=0.03 if rfi else 0.0,
                     rfi_amp=60.0 if nbits == 8 else 6000.0,
                     pulses=[(0.4 * dmh, 0.3 * n * 64e-6, 2e-4, 30.0 if nbits == 8 else 3000.0)])
    x, hdr = make_chunk(spec)
    for k in ("tsamp", "fch1", "foff"):
        hdr[k] = float(F32(hdr[k]))
    lo = float(F32(hdr["fch1"]))
    hi = float(F32(F32(hdr["fch1"]) + F32(nchans - 1) * F32(hdr["foff"])))
    r = RfiParams(use_zero_dm=True, use_iqrm=True,
                  iqrm=IqrmParams(mode=0, radius_frac=0.05, nsigma=3.0, win_sec=0.1, hop_sec=0.05)) if rfi else None
    if algo == "brute":
        plan = Plan(hdr, 0.0, dmh, lo, hi, step, ds, n * hdr["tsamp"] * 0.3, algorithm="brute",
                    freq_mode="fil")
    else:
        plan = Plan(hdr, 0.0, dmh, lo, hi, step, ds, algorithm="subband", subband_width=sbw, rfi=r)
    return plan, dev(x)


@pytest.mark.parametrize("use_graph,persistent", [(True, False), (False, False), (True, True),
                                                   (False, True)])
def test_batch_equals_individual_runs(use_graph, persistent):
    items = [make(c, 40 + i) for i, c in enumerate(CHUNKS)]
    plans = [p for p, _ in items]
    xs = [x for _, x in items]
    want = [to_np(p.run(x)) for p, x in items]
    torch.cuda.synchronize()
    batch = Batch(plans, use_graph=use_graph, persistent=persistent)
    outs = batch.empty_outputs()
    for rep in range(3):  # replays of the same buffers
        for o in outs:
            o.fill_(0)
        batch.run(xs, outs)
        batch.status()
        for i, (o, w) in enumerate(zip(outs, want)):
            assert np.array_equal(to_np(o), w), f"chunk {i} differs (run {rep})"
    info = batch.info
    assert info["nplans"] == len(CHUNKS) and info["graph"] == int(use_graph)
    assert info["persistent"] == int(persistent) and info["sum_launches"] >= 1
    assert info["graph_captures"] == (1 if use_graph else 0)
    # new output buffers: one more capture, same results
    outs2 = batch.empty_outputs()
    batch.run(xs, outs2)
    batch.status()
    for o, w in zip(outs2, want):
        assert np.array_equal(to_np(o), w)
    assert batch.info["graph_captures"] == (2 if use_graph else 0)
    batch.close()


@pytest.mark.parametrize("persistent", [False, True])
def test_batch_runs_own_kernels_for_32bit_plans(persistent):
    """A 32-bit plan (direct-load kernels) next to staged plans: all results exact."""
    rng = np.random.default_rng(0)
    hdr = dict(tsamp=1e-4, fch1=1200.0, foff=1.0, nbits=32, nchans=64, ndata=2048)
    x32 = rng.integers(0, 1 << 20, size=(2048, 64)).astype(np.uint32)
    p32 = Plan(hdr, 0.0, 50.0, 1200.0, 1263.0, 1.0, 1, algorithm="subband")
    d32 = torch.from_numpy(x32.view(np.int32)).cuda().view(torch.uint32)
    p8, x8 = make(CHUNKS[0], 1)
    want32 = p32.run(d32).view(torch.int64).cpu().numpy()
    want8 = to_np(p8.run(x8))
    batch = Batch([p32, p8], persistent=persistent)
    o32, o8 = batch.run([d32, x8])
    batch.status()
    assert batch.info["own_plans"] == 1
    assert np.array_equal(o32.view(torch.int64).cpu().numpy(), want32)
    assert np.array_equal(to_np(o8), want8)
    with pytest.raises(ValueError, match="twice"):
        Batch([p8, p8])
