"""Host-buffer runs queued one after another (dd_run_host_async / dd_run_host_join):
consecutive chunks overlap one chunk's output copy with the next one's input
copy, and the next chunk's sums wait for the copy of the output they overwrite.
Each result must equal the device-resident run of the same chunk bit for bit,
across several time tiles (whose outputs travel while later tiles are summed)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import Plan  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


def pinned(shape, np_dtype):
    t = {np.uint8: torch.uint8, np.uint32: torch.int32}[np_dtype]
    a = torch.empty(shape, dtype=t, pin_memory=True).numpy()
    return a if np_dtype == np.uint8 else a.view(np.uint32)


def chunks(nchans, nsamp, seeds):
    out = []
    for s in seeds:
        spec = ChunkSpec(nchans=nchans, nsamp=nsamp, nbits=8, seed=s, rfi_frac=0.05, impulses=4,
                         pulses=[(300.0 + 100 * s, 0.2, 2e-4, 25.0)])
        x, _ = make_chunk(spec)
        h = pinned(x.shape, np.uint8)
        h[...] = x
        out.append((spec, h))
    return out


def header(spec):
    hdr = dict(tsamp=float(F32(spec.tsamp)), fch1=float(F32(spec.fch1)), foff=float(F32(spec.foff)),
               nbits=8, nchans=spec.nchans, ndata=spec.nsamp)
    freq = O.freq_table_header(hdr["fch1"], hdr["foff"], spec.nchans)
    return hdr, float(F32(freq[0])), float(F32(freq[-1]))


def device_result(plan, x):
    return plan.run(torch.from_numpy(x).cuda()).view(torch.int32).cpu().numpy().view(np.uint32)


def test_queued_subband_runs_across_tiles_equal_device_runs():
    cs = chunks(4096, 1 << 16, (1, 2, 3))
    hdr, fs, fe = header(cs[0][0])
    plan = Plan(hdr, 0.0, 3000.0, fs, fe, 0.5, 1, algorithm="subband", subband_width=64)
    ntiles = -(-plan.info["out_cols"] // plan.info["tile_samples"])
    assert ntiles >= 2, f"{ntiles} time tiles"
    want = [device_result(plan, x) for _, x in cs]
    outs = [pinned(plan.out_shape, np.uint32) for _ in cs]
    stream = torch.cuda.current_stream()
    for (_, x), o in zip(cs, outs):
        plan.run_host_async(x, o, stream)
    plan.run_host_join(stream, sync=True)
    for o, w in zip(outs, want):
        assert np.array_equal(o, w)
    # a blocking host run after queued ones, into a fresh buffer
    assert np.array_equal(plan.run_host(cs[1][1]), want[1])
    plan.close()


def test_queued_brute_force_runs_equal_device_runs():
    cs = chunks(512, 1 << 15, (4, 5))
    spec = cs[0][0]
    hdr = dict(tsamp=1e-4, fch1=1200.0, foff=0.5, nbits=8, nchans=512, ndata=spec.nsamp)
    freq = O.freq_table_fil(1200.0, 0.5, 512)
    fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
    plan = Plan(hdr, 0.0, 400.0, fs, fe, 1.0, 1, 0.5, algorithm="brute", freq_mode="fil")
    want = [device_result(plan, x) for _, x in cs]
    outs = [pinned(plan.out_shape, np.uint32) for _ in cs]
    stream = torch.cuda.current_stream()
    for (_, x), o in zip(cs, outs):
        plan.run_host_async(x, o, stream)
    plan.run_host_join(stream, sync=True)
    for o, w in zip(outs, want):
        assert np.array_equal(o, w)
    plan.close()


def test_queued_run_rejects_mismatched_output():
    cs = chunks(256, 8192, (6,))
    hdr, fs, fe = header(cs[0][0])
    plan = Plan(hdr, 0.0, 300.0, fs, fe, 1.0, 1, algorithm="subband")
    bad = np.empty((plan.out_shape[0], plan.out_shape[1] - 1), np.uint32)
    with pytest.raises(ValueError, match="output must be"):
        plan.run_host_async(cs[0][1], bad)
    plan.close()
