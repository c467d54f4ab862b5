"""Streams (dd_stream_*): a beam pushed chunk by chunk equals the plain call.

Without RFI stages the pushes concatenate to the plain call on the whole beam
behind a zero tail (every output column reads only samples inside its push's
buffer).  With RFI stages each push equals the plain call on its own buffer
[tail | chunk], first chunk/ds columns (the definition of a streamed chunk)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import IqrmParams, Plan, RfiParams, Stream  # noqa: E402
from astroflow_b200.synth import ChunkSpec, make_chunk  # noqa: E402

F32 = np.float32


def to_np(t):
    return t.view(torch.int32).cpu().numpy().view(np.uint32)


def dev(x):
    x = np.ascontiguousarray(x)
    if x.dtype == np.uint16:
        return torch.from_numpy(x.view(np.int16)).cuda().view(torch.uint16)
    return torch.from_numpy(x).cuda()


CASES = [
    # nchans, nbits, chunk, nchunks, dm_high, dm_step, ds, sbw
    (256, 8, 3000, 5, 400.0, 1.0, 1, 32),
    (512, 16, 2048, 4, 300.0, 0.5, 2, 64),
    (128, 8, 1000, 6, 800.0, 2.0, 4, 16),
]


def beam(case, seed):
    nchans, nbits, chunk, k, dmh, step, ds, sbw = case
    spec = ChunkSpec(nchans=nchans, nsamp=chunk * k, nbits=nbits, tsamp=64e-6, seed=seed,
                     rfi_frac=0.04, rfi_amp=60.0 if nbits == 8 else 6000.0, impulses=3,
                     imp_amp=50.0 if nbits == 8 else 5000.0,
                     pulses=[(0.5 * dmh, 0.4 * chunk * k * 64e-6, 2e-4, 40.0 if nbits == 8 else 4000.0)])
    x, hdr = make_chunk(spec)
    for key in ("tsamp", "fch1", "foff"):
        hdr[key] = float(F32(hdr[key]))
    lo = float(F32(hdr["fch1"]))
    hi = float(F32(F32(hdr["fch1"]) + F32(nchans - 1) * F32(hdr["foff"])))
    return x, hdr, lo, hi


@pytest.mark.parametrize("case", CASES)
def test_stream_equals_plain_call_on_the_beam(case):
    nchans, nbits, chunk, k, dmh, step, ds, sbw = case
    x, hdr, lo, hi = beam(case, 7)
    h1 = dict(hdr, ndata=chunk)
    s = Stream(h1, 0.0, dmh, lo, hi, step, ds, subband_width=sbw)
    info = s.info
    tail = info["tail_samples"]
    assert tail % ds == 0 and info["out_cols"] == chunk // ds and info["chunk_samples"] == chunk
    outs = [to_np(s.push(dev(x[i * chunk:(i + 1) * chunk]))) for i in range(k)]
    assert s.info["pushed_samples"] == k * chunk
    padded = np.concatenate([np.zeros((tail, nchans), x.dtype), x])
    full = Plan(dict(hdr, ndata=padded.shape[0]), 0.0, dmh, lo, hi, step, ds, subband_width=sbw)
    want = to_np(full.run(dev(padded)))[:, :k * chunk // ds]
    assert np.array_equal(np.concatenate(outs, axis=1), want)


@pytest.mark.parametrize("case", CASES[:2])
def test_stream_push_equals_plain_call_on_its_buffer_with_rfi(case):
    nchans, nbits, chunk, k, dmh, step, ds, sbw = case
    x, hdr, lo, hi = beam(case, 9)
    rfi = RfiParams(use_zero_dm=True, use_iqrm=True, use_mask=True,
                    iqrm=IqrmParams(mode=0, radius_frac=0.05, nsigma=3.0, win_sec=0.05, hop_sec=0.03))
    s = Stream(dict(hdr, ndata=chunk), 0.0, dmh, lo, hi, step, ds, subband_width=sbw, rfi=rfi,
               bad_channels=[3, 10], zero_dm_mode="range")
    tail = s.info["tail_samples"]
    buf = np.zeros((tail + chunk, nchans), x.dtype)
    plain = Plan(dict(hdr, ndata=tail + chunk), 0.0, dmh, lo, hi, step, ds, subband_width=sbw,
                 rfi=rfi, bad_channels=[3, 10], zero_dm_mode="range")
    for i in range(k):
        buf[tail:] = x[i * chunk:(i + 1) * chunk]
        got = to_np(s.push(dev(x[i * chunk:(i + 1) * chunk])))
        want = to_np(plain.run(dev(buf)))[:, :chunk // ds]
        assert np.array_equal(got, want), f"push {i}"
        buf[:tail] = buf[chunk:].copy()


def test_stream_rejects_ragged_chunks():
    x, hdr, lo, hi = beam(CASES[0], 1)
    with pytest.raises(ValueError):
        Stream(dict(hdr, ndata=1001), 0.0, 100.0, lo, hi, 1.0, 2)
