"""The image step on the GPU (dd_images; include/data.h:620-727 and 299-369)
against OpenCV run on the host on the same sums: the float resize
(INTER_AREA / INTER_LANCZOS4) bit for bit, and the 512x512x3 viridis images
byte for byte.  One documented exception: an area resize whose scales are both
integers with a horizontal factor other than 2 or 4 sums its blocks in an order
OpenCV does not publish; there the float resize is checked to 1e-6 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
cv2 = pytest.importorskip("cv2")
from astroflow_b200 import postprocess  # noqa: E402
from oracle import cv2_images as CVI  # noqa: E402


def _dev(a: np.ndarray):
    view = {np.uint32: (np.int32, torch.uint32), np.uint64: (np.int64, torch.uint64)}[a.dtype.type]
    return torch.from_numpy(a.view(view[0])).cuda().view(view[1])


SHAPES = [
    # rows, slice widths, dtype, value scale
    (6001, [10172, 10172, 3000], np.uint32, 1e6),     # area, general scales (headline slices)
    (301, [2000, 700], np.uint32, 4e4),               # Lanczos: rows up, columns down
    (1024, [1024, 2048], np.uint32, 1e6),             # area, integer scales 2x2 and 2x4
    (1536, [1536], np.uint32, 1e6),                   # area, integer 3x3 (order unpublished)
    (700, [512, 300], np.uint64, 3e9),                # Lanczos with 64-bit sums above 2^24
    (2, [900], np.uint32, 100.0),                     # two rows
    (1, [900], np.uint32, 100.0),                     # one row
    (600, [20000], np.uint32, 5e5),                   # slice wider than the staged row
]


@pytest.mark.parametrize("rows,widths,dt,scale", SHAPES)
def test_resize_and_images_match_opencv(rows, widths, dt, scale):
    rng = np.random.default_rng(rows)
    cols = sum(widths) + 17
    raw = (rng.random((rows, cols)) * scale).astype(dt)
    starts = list(np.cumsum([0] + widths[:-1]) + 5)
    d = _dev(raw)
    got = postprocess.device_images(d, starts, widths, resized=True).cpu().numpy()
    imgs = postprocess.device_images(d, starts, widths).cpu().numpy()
    for i, (s, w) in enumerate(zip(starts, widths)):
        f = np.ascontiguousarray(raw[:, s:s + w], dtype=np.float32)
        interp = cv2.INTER_AREA if (rows > 512 and w > 512) else cv2.INTER_LANCZOS4
        want = cv2.resize(f, (512, 512), interpolation=interp)
        integer = interp == cv2.INTER_AREA and rows % 512 == 0 and w % 512 == 0
        if integer and (w // 512) not in (2, 4):
            np.testing.assert_allclose(got[i], want, rtol=1e-6, atol=0)
        else:
            np.testing.assert_array_equal(got[i], want)
            np.testing.assert_array_equal(imgs[i], CVI.image(raw[:, s:s + w]))


def test_constant_sums():
    """A constant slice whose resize stays exactly constant maps to the first
    color (zero scale); one whose area weights round unevenly is stretched over
    the whole map, as OpenCV does."""
    raw = np.full((1024, 1024), 7, np.uint32)
    img = postprocess.device_images(_dev(raw), [0], [1024]).cpu().numpy()[0]
    assert (img == postprocess.viridis_lut()[0]).all()
    raw = np.full((800, 1500), 7, np.uint32)
    img = postprocess.device_images(_dev(raw), [0], [1500]).cpu().numpy()[0]
    np.testing.assert_array_equal(img, CVI.image(raw))


def test_slice_images_on_device_equal_host():
    rng = np.random.default_rng(1)
    raw = rng.integers(0, 1 << 20, (3001, 25000)).astype(np.uint32)
    want = CVI.slice_images(raw, 64e-6, 2, 0.5)
    got = postprocess.device_slice_images(_dev(raw), 64e-6, 2, 0.5)
    assert len(got) == len(want) == 7
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


def test_host_images_outlive_the_staging_block():
    """Images come to the host through one reused pinned block; each call's arrays
    are its own and keep their bytes when the next call (fewer or more images)
    reuses the block."""
    rng = np.random.default_rng(5)
    raws = [rng.integers(0, 1 << 16, (700, c)).astype(np.uint32) for c in (2600, 900, 4100)]
    results = [postprocess.device_slice_images(_dev(r), 1e-3, 1, 0.5) for r in raws]
    for r, got in zip(raws, results):
        want = CVI.slice_images(r, 1e-3, 1, 0.5)
        assert len(got) == len(want)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)


def test_bad_arguments_raise():
    raw = _dev(np.zeros((10, 100), np.uint32))
    with pytest.raises(ValueError):
        postprocess.device_images(raw, [90], [20])
    with pytest.raises(ValueError):
        postprocess.device_images(raw, [0], [0])
