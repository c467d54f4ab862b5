"""Ingest into device memory: SIGPROC filterbank files and host arrays, in the
layout the plans read ([time][channel], ascending frequency).

The reference reads a filterbank file into host memory and reverses its channels
on the host when foff < 0 (src/data/filterbank.cpp:454-473, 793-842); its PSRFITS
reader averages polarisations 0 and 1 and flips the band in numpy
(python/astroflow/io/psrfits.py:31-80).  Here pinned staging blocks are filled by
worker threads and copied block by block, with the flip and the polarisation
average done on the device (dd_fil_read, dd_ingest_host).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import _lib


class FilHeader(ctypes.Structure):
    _fields_ = [("tsamp", ctypes.c_double), ("fch1", ctypes.c_double), ("foff", ctypes.c_double),
                ("tstart", ctypes.c_double), ("ndata", ctypes.c_int64),
                ("header_bytes", ctypes.c_int64), ("nbits", ctypes.c_int32),
                ("nchans", ctypes.c_int32), ("nifs", ctypes.c_int32), ("flipped", ctypes.c_int32),
                ("has_freq_table", ctypes.c_int32), ("pad", ctypes.c_int32)]


FLIP = 1
SIGNED = 2
_TORCH = {1: "uint8", 2: "uint16", 4: "uint32"}


def _bind(L):
    if getattr(L, "_ingest_bound", False):
        return
    L.dd_fil_read_header.argtypes = [ctypes.c_char_p, ctypes.POINTER(FilHeader), ctypes.c_void_p,
                                     ctypes.c_int32]
    L.dd_fil_read.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                              ctypes.c_void_p]
    L.dd_ingest_host.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                 ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    for f in (L.dd_fil_read_header, L.dd_fil_read, L.dd_ingest_host):
        f.restype = ctypes.c_int
    L._ingest_bound = True


def fil_header(path: str) -> Tuple[dict, np.ndarray]:
    """The file's header as the reference's Filterbank reports it after its
    channel flip, and its frequency table (ascending)."""
    L = _lib.load()
    _bind(L)
    h = FilHeader()
    _lib.check(L.dd_fil_read_header(str(path).encode(), ctypes.byref(h), None, 0))
    table = np.zeros(h.nchans, np.float64)
    _lib.check(L.dd_fil_read_header(str(path).encode(), ctypes.byref(h), table.ctypes.data,
                                    h.nchans))
    return {n: getattr(h, n) for n, _ in FilHeader._fields_ if n != "pad"}, table


def read_filterbank(path: str, t0: int = 0, nsamp: Optional[int] = None, device: int = 0,
                    stream=None):
    """Samples [t0, t0 + nsamp) of a single-IF SIGPROC file as a device tensor
    [nsamp, nchans] (uint8/16/32) in ascending channel order, with the header and
    frequency table of fil_header."""
    import torch

    L = _lib.load()
    hdr, table = fil_header(path)
    n = hdr["ndata"] - t0 if nsamp is None else int(nsamp)
    dt = getattr(torch, _TORCH[hdr["nbits"] // 8])
    out = torch.empty((max(n, 0), hdr["nchans"]), dtype=dt, device=f"cuda:{device}")
    if stream is None:
        stream = torch.cuda.current_stream(out.device)
    with torch.cuda.device(out.device):
        _lib.check(L.dd_fil_read(str(path).encode(), int(t0), int(n), ctypes.c_void_p(out.data_ptr()),
                                 ctypes.c_void_p(stream.cuda_stream)))
    return out, hdr, table


def to_device(a: np.ndarray, flip: bool = False, device: int = 0, stream=None):
    """A host array [nsamp, nchans] (or [nsamp, npol, nchans]: polarisations 0 and 1
    averaged as the reference's PSRFITS reader does) copied through pinned
    staging into a device tensor [nsamp, nchans], channels reversed if flip."""
    import torch

    L = _lib.load()
    _bind(L)
    a = np.asarray(a)
    if not a.dtype.isnative:
        a = a.astype(a.dtype.newbyteorder("="))
    a = np.ascontiguousarray(a)
    if a.dtype.kind not in "ui" or a.dtype.itemsize not in (1, 2, 4):
        raise ValueError("samples must be 8-, 16- or 32-bit integers")
    if a.ndim == 2:
        nsamp, npol, nchans = a.shape[0], 1, a.shape[1]
    elif a.ndim == 3:
        nsamp, npol, nchans = a.shape
    else:
        raise ValueError("expected [nsamp, nchans] or [nsamp, npol, nchans]")
    dt = getattr(torch, ("int" if a.dtype.kind == "i" else "uint") + str(8 * a.dtype.itemsize))
    out = torch.empty((nsamp, nchans), dtype=dt, device=f"cuda:{device}")
    if stream is None:
        stream = torch.cuda.current_stream(out.device)
    flags = (FLIP if flip else 0) | (SIGNED if a.dtype.kind == "i" else 0)
    with torch.cuda.device(out.device):
        _lib.check(L.dd_ingest_host(a.ctypes.data, nsamp, npol, nchans, a.dtype.itemsize, flags,
                                    ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_void_p(stream.cuda_stream)))
    return out
