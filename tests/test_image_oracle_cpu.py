"""The image step's arithmetic pinned on the CPU: the oracle's numpy restatement of
the area and Lanczos-4 resizes and of the min-max normalisation equals OpenCV
(the library the reference calls, include/data.h:620-727) bit for bit.  The GPU
kernels (dd_images) follow the same operations; tests/test_gpu_images.py checks
them against cv2 on the GPU."""
import numpy as np
import pytest

from oracle import oracle as O

cv2 = pytest.importorskip("cv2")


@pytest.mark.parametrize("shape", [(1000, 1500), (600, 700), (1024, 10172), (513, 513)])
def test_area_resize_matches_opencv(shape):
    src = (np.random.default_rng(shape[0]).random(shape) * 1e6).astype(np.float32)
    want = cv2.resize(src, (512, 512), interpolation=cv2.INTER_AREA)
    np.testing.assert_array_equal(O.resize_area(src), want)


@pytest.mark.parametrize("shape", [(301, 2000), (100, 700), (600, 300), (512, 512), (2, 900), (1, 900)])
def test_lanczos4_resize_matches_opencv(shape):
    src = (np.random.default_rng(shape[1]).random(shape) * 1e6).astype(np.float32)
    want = cv2.resize(src, (512, 512), interpolation=cv2.INTER_LANCZOS4)
    np.testing.assert_array_equal(O.resize_lanczos4(src), want)


def test_normalize_matches_opencv():
    rng = np.random.default_rng(7)
    for k in range(40):
        img = (rng.random((64, 64)) * rng.choice([1, 1e3, 1e6, 3e8]) + rng.choice([0, 5, 1e5]))
        img = img.astype(np.float32)
        want = cv2.normalize(img, None, 0, 255, cv2.NORM_MINMAX, cv2.CV_8U)
        np.testing.assert_array_equal(O.normalize_u8(img), want)
    flat = np.full((8, 8), 7.0, np.float32)
    assert (O.normalize_u8(flat) == cv2.normalize(flat, None, 0, 255, cv2.NORM_MINMAX, cv2.CV_8U)).all()
