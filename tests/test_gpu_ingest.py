"""Ingest on the GPU (dd_fil_read, dd_ingest_host): the device tensor equals what
the reference's host readers produce (src/data/filterbank.cpp:454-473 and
793-842; python/astroflow/io/psrfits.py:31-80), across sample widths, channel
orders, windows and multi-block transfers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from astroflow_b200 import _astroflow_core as C  # noqa: E402
from astroflow_b200 import ingest  # noqa: E402
from sigproc_writer import write_fil  # noqa: E402

DT = {8: np.uint8, 16: np.uint16, 32: np.uint32}


def host(t):
    view = {torch.uint8: (torch.uint8, np.uint8), torch.uint16: (torch.int16, np.uint16),
            torch.uint32: (torch.int32, np.uint32), torch.int16: (torch.int16, np.int16),
            torch.int8: (torch.int8, np.int8), torch.int32: (torch.int32, np.int32)}[t.dtype]
    return t.view(view[0]).cpu().numpy().view(view[1])


@pytest.mark.parametrize("nbits,nsamp,nchans,foff", [
    (8, 30000, 4096, -0.122), (16, 5000, 1000, 0.5), (32, 3000, 777, -1.0), (8, 7, 3, -1.0)])
def test_read_filterbank_equals_host_reader(nbits, nsamp, nchans, foff, tmp_path):
    rng = np.random.default_rng(nbits + nsamp)
    raw = rng.integers(0, np.iinfo(DT[nbits]).max, (nsamp, nchans), dtype=DT[nbits])
    p = str(tmp_path / "a.fil")
    write_fil(p, raw, 64e-6, 1500.0, foff)
    want = C.Filterbank(p).data[:, 0, :]
    x, hdr, table = ingest.read_filterbank(p)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(x), want)
    assert hdr["flipped"] == int(foff < 0)
    t0, n = nsamp // 3, nsamp // 2
    x2, _, _ = ingest.read_filterbank(p, t0, n)
    np.testing.assert_array_equal(host(x2), want[t0:t0 + n])


def test_read_errors(tmp_path):
    p = str(tmp_path / "a.fil")
    write_fil(p, np.zeros((10, 8), np.uint8), 1e-4, 1000.0, 1.0)
    with pytest.raises(ValueError, match="outside the file"):
        ingest.read_filterbank(p, 5, 10)


@pytest.mark.parametrize("dt,npol,flip", [
    (np.uint8, 2, True), (np.uint8, 4, False), (np.uint16, 2, True), (np.int16, 2, True),
    (np.uint8, 1, True), (np.uint16, 1, False)])
def test_host_arrays_and_polarisation_average(dt, npol, flip):
    rng = np.random.default_rng(npol)
    info = np.iinfo(dt)
    a = rng.integers(info.min, info.max, (20000, npol, 512), dtype=dt)
    if npol >= 2:   # psrfits.py:49: ((a + b) / 2).astype(dtype) with numpy's wrapping sum
        want = ((a[:, 0, :] + a[:, 1, :]) / 2).astype(dt)
    else:
        want = a[:, 0, :]
    if flip:
        want = np.flip(want, axis=1)
    got = ingest.to_device(a if npol > 1 else a[:, 0, :], flip=flip)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(got), want)


def test_big_endian_input():
    a = np.arange(2 * 3 * 40, dtype=">u2").reshape(40, 3 * 2)
    got = ingest.to_device(a)
    np.testing.assert_array_equal(host(got), a.astype(np.uint16))
