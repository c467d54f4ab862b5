"""DM-time images for the detector, as the reference builds them after dedispersion.

The reference converts the raw DM x time sums into 512x512 viridis images before
returning to Python: include/data.h:620-727 (the GPU paths: cut the columns into
slices of t_sample seconds) and include/data.h:299-369 (the CPU path: one image
per slice it already produced).  Each image is: uint sums -> float32, resize to
512x512 (INTER_AREA when both dimensions exceed 512, else INTER_LANCZOS4),
min-max normalise to uint8, gray -> RGB, COLORMAP_VIRIDIS.  Here the GPU does all
of it through dd_images (device_slice_images, device_images): it resizes,
normalises and colors in device memory, and only the images come to the host.
"""
from __future__ import annotations

import threading
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Sequence

import numpy as np

TARGET = 512


def samples_per_slice(tsamp: float, time_downsample: int, slice_duration: float) -> int:
    """include/data.h:645-647: (size_t)(slice_duration / (tsamp * time_downsample)) in float."""
    ts = np.float32(np.float32(tsamp) * np.float32(time_downsample))
    return int(np.float32(slice_duration) / ts)


_LUT: Optional[np.ndarray] = None


def viridis_lut() -> np.ndarray:
    """The 256 BGR colors OpenCV's COLORMAP_VIRIDIS gives a gray ramp converted to
    RGB (the reference's cvtColor + applyColorMap), as a [256, 3] uint8 table."""
    global _LUT
    if _LUT is None:
        import cv2

        ramp = np.arange(256, dtype=np.uint8).reshape(16, 16)
        rgb = cv2.cvtColor(ramp, cv2.COLOR_GRAY2RGB)
        _LUT = np.ascontiguousarray(cv2.applyColorMap(rgb, cv2.COLORMAP_VIRIDIS).reshape(256, 3))
    return _LUT


def device_images(out, col_start: Sequence[int], col_count: Sequence[int], target: int = TARGET,
                  stream=None, resized: bool = False):
    """Images of column slices of a device DM-time tensor out [rows, cols] (uint32
    or uint64), made on the GPU (dd_images).  Returns the device tensor
    [n, target, target, 3] uint8, or with resized=True the float images
    [n, target, target] before normalisation."""
    import ctypes

    import torch

    from . import _lib

    L = _lib.load()
    if not out.is_cuda or out.dim() != 2 or out.element_size() not in (4, 8):
        raise ValueError("out must be a 2-D CUDA tensor of uint32 or uint64 sums")
    if out.stride(1) != 1:
        raise ValueError("out rows must be contiguous")
    c0 = np.ascontiguousarray(col_start, np.int64)
    cn = np.ascontiguousarray(col_count, np.int64)
    n = int(c0.size)
    dev = out.device
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    img = f32 = None
    if resized:
        f32 = torch.empty((n, target, target), dtype=torch.float32, device=dev)
    else:
        img = torch.empty((n, target, target, 3), dtype=torch.uint8, device=dev)
    lut = viridis_lut()
    _lib.check(L.dd_images(ctypes.c_void_p(out.data_ptr()), out.element_size(), out.shape[0],
                           out.stride(0), n, c0.ctypes.data, cn.ctypes.data, target,
                           lut.ctypes.data, None if img is None else img.data_ptr(),
                           None if f32 is None else f32.data_ptr(),
                           ctypes.c_void_p(stream.cuda_stream)))
    return f32 if resized else img


def slice_bounds(cols: int, sps: int):
    """Column starts and widths of the t_sample slices (include/data.h:644-691)."""
    n = (cols + sps - 1) // sps
    starts = [i * sps for i in range(n)]
    return starts, [min(sps, cols - s) for s in starts]


# One pinned block, kept for the life of the process and grown on demand, through
# which images come to the host: pinning a fresh block per call (the returned
# arrays outlive the call) cost 80-700 ms for 82 MB of images on a busy host, a
# copy from the device into pageable memory about 35 ms.
_STAGE = None
_STAGE_LOCK = threading.Lock()
_COPY_POOL: Optional[ThreadPoolExecutor] = None


def to_host_images(dev_imgs) -> List[np.ndarray]:
    """[n, t, t, 3] device images as n host arrays (views of one new block): one
    device-to-host copy into the pinned staging block, then a parallel host copy
    into the returned block."""
    import torch

    global _STAGE, _COPY_POOL
    if dev_imgs.dtype != torch.uint8:
        raise ValueError("images must be uint8")
    n = int(dev_imgs.shape[0])
    if n == 0:
        return []
    out = np.empty(tuple(dev_imgs.shape), np.uint8)
    nbytes = dev_imgs.numel() * dev_imgs.element_size()
    with _STAGE_LOCK:
        if _STAGE is None or _STAGE.numel() < nbytes:
            _STAGE = None
            _STAGE = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        if _COPY_POOL is None:
            _COPY_POOL = ThreadPoolExecutor(max_workers=8)
        stage = _STAGE[:nbytes].view(tuple(dev_imgs.shape))
        stage.copy_(dev_imgs.contiguous())  # synchronous: returns once the bytes are on the host
        src = stage.numpy()
        step = max(1, (n + 7) // 8)
        list(_COPY_POOL.map(lambda i: np.copyto(out[i:i + step], src[i:i + step]),
                            range(0, n, step)))
    return [out[i] for i in range(n)]


def device_slice_images(out, tsamp: float, time_downsample: int,
                        slice_duration: float) -> List[np.ndarray]:
    """The images of the t_sample-second slices of a device DM-time tensor (include/data.h:620-727)."""
    sps = samples_per_slice(tsamp, time_downsample, slice_duration)
    if sps <= 0:
        raise ValueError("t_sample is shorter than one (downsampled) sample")
    starts, counts = slice_bounds(out.shape[1], sps)
    return to_host_images(device_images(out, starts, counts))
