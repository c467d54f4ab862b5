"""Argument checks of the allocation-free IQRM wrapper (iqrm_masks_noalloc).

The C entry point writes max_windows x nchans mask bytes and 2 x max_windows
bound words into caller-owned buffers, so the Python wrapper must refuse any
buffer that is too small, of the wrong type or layout, or not on the current
GPU before the call reaches the device.  Each case below breaks one rule; none
needs a GPU because every rejection happens before the library is called.
"""
import pytest

torch = pytest.importorskip("torch")
from astroflow_b200.dedisp import IqrmParams, iqrm_masks_noalloc  # noqa: E402

NCH = 16
IQ = IqrmParams(mode=0, radius_frac=0.1, nsigma=3.0, win_sec=0.0, hop_sec=0.0)


def good():
    return dict(x=torch.zeros((100, NCH), dtype=torch.uint8),
                masks=torch.zeros((2, NCH), dtype=torch.uint8),
                bounds=torch.zeros((2, 2), dtype=torch.int32))


CASES = [
    ("nchans", dict(nchans=0), "nchans"),
    ("x dtype", dict(x=torch.zeros((100, NCH), dtype=torch.float32)), "8-, 16- or 32-bit"),
    ("x ragged", dict(x=torch.zeros((100 * NCH + 3,), dtype=torch.uint8)), "whole"),
    ("x strided", dict(x=torch.zeros((NCH, 100), dtype=torch.uint8).t()), "contiguous"),
    ("masks dtype", dict(masks=torch.zeros((2, NCH), dtype=torch.int32)), "masks"),
    ("masks narrow", dict(masks=torch.zeros((2, NCH - 1), dtype=torch.uint8)), "masks"),
    ("masks 1-D", dict(masks=torch.zeros((2 * NCH,), dtype=torch.uint8)), "masks"),
    ("bounds short", dict(bounds=torch.zeros((1, 2), dtype=torch.int32)), "bounds"),
    ("bounds cols", dict(bounds=torch.zeros((2, 3), dtype=torch.int32)), "bounds"),
    ("bounds dtype", dict(bounds=torch.zeros((2, 2), dtype=torch.int64)), "bounds"),
    ("band", dict(chan_start=5, chan_end=5), "channel range"),
    ("band past end", dict(chan_end=NCH + 1), "channel range"),
    ("host tensors", dict(), "current CUDA device"),
]


@pytest.mark.parametrize("name,change,msg", CASES, ids=[c[0] for c in CASES])
def test_noalloc_wrapper_rejects(name, change, msg):
    a = good()
    a.update(nchans=NCH, chan_start=0, chan_end=NCH - 1)
    a.update(change)
    with pytest.raises(ValueError, match=msg):
        iqrm_masks_noalloc(a["x"], a["nchans"], a["chan_start"], a["chan_end"], 1e-4, IQ,
                           a["masks"], a["bounds"])
