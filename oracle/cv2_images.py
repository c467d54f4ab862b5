"""ORACLE — test infrastructure, not product code.

The reference's image step run with OpenCV itself, the library the reference
calls: include/data.h:620-727 (the GPU paths cut the raw [dm, time] sums into
slices of t_sample seconds) and include/data.h:299-369 (the CPU path images the
slices it already produced).  Each image: uint sums -> float32, resize to
512x512 (INTER_AREA when both dimensions exceed 512, else INTER_LANCZOS4),
min-max normalise to uint8, gray -> RGB, COLORMAP_VIRIDIS.  Only tests/ import
this module, as the oracle of the library's GPU image step (dd_images).
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor
from typing import List, Sequence

import numpy as np

TARGET = 512


def image(block: np.ndarray, target: int = TARGET) -> np.ndarray:
    """One slice's image (include/data.h:688-727)."""
    import cv2

    f = np.ascontiguousarray(block, dtype=np.float32)
    rows, cols = f.shape
    interp = cv2.INTER_AREA if (rows > target and cols > target) else cv2.INTER_LANCZOS4
    resized = cv2.resize(f, (target, target), interpolation=interp)
    norm = cv2.normalize(resized, None, 0, 255, cv2.NORM_MINMAX, cv2.CV_8U)
    rgb = cv2.cvtColor(norm, cv2.COLOR_GRAY2RGB)
    return np.ascontiguousarray(cv2.applyColorMap(rgb, cv2.COLORMAP_VIRIDIS))


def samples_per_slice(tsamp: float, time_downsample: int, slice_duration: float) -> int:
    """include/data.h:645-647: (size_t)(slice_duration / (tsamp * time_downsample)) in float."""
    ts = np.float32(np.float32(tsamp) * np.float32(time_downsample))
    return int(np.float32(slice_duration) / ts)


def slice_images(raw: np.ndarray, tsamp: float, time_downsample: int, slice_duration: float,
                 threads: int = 16) -> List[np.ndarray]:
    """Images of consecutive column slices of raw [dm, time] sums (include/data.h:620-727)."""
    sps = samples_per_slice(tsamp, time_downsample, slice_duration)
    if sps <= 0:
        raise ValueError("t_sample is shorter than one (downsampled) sample")
    cols = raw.shape[1]
    n = (cols + sps - 1) // sps
    blocks = [raw[:, i * sps:min((i + 1) * sps, cols)] for i in range(n)]
    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        return list(ex.map(image, blocks))


def images(blocks: Sequence[np.ndarray], threads: int = 16) -> List[np.ndarray]:
    """One image per block (include/data.h:299-369)."""
    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        return list(ex.map(image, blocks))
