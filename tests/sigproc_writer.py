"""Writes small SIGPROC filterbank files for the tests (the format read by
src/data/filterbank.cpp:319-452: length-prefixed keyword strings, int32 and
float64 values, HEADER_START ... HEADER_END, then samples time-major)."""
import struct

import numpy as np

_INT = {"telescope_id", "machine_id", "data_type", "barycentric", "pulsarcentric", "nbits",
        "nchans", "nifs", "nbins", "ibeam", "nbeams", "npuls", "nsamples"}


def _s(text: str) -> bytes:
    b = text.encode()
    return struct.pack("<i", len(b)) + b


def write_fil(path, data: np.ndarray, tsamp: float, fch1: float, foff: float, tstart=60000.0,
              freq_table=None, extra=(), source_name="synthetic"):
    """data: [nsamp, nchans] uint8/16/32 in file channel order."""
    data = np.ascontiguousarray(data)
    nbits = data.dtype.itemsize * 8
    nsamp, nchans = data.shape
    out = [_s("HEADER_START"), _s("source_name"), _s(source_name)]

    def kv(key, val):
        out.append(_s(key))
        out.append(struct.pack("<i" if key in _INT else "<d", val))

    kv("telescope_id", 0)
    kv("machine_id", 0)
    kv("data_type", 1)
    kv("tstart", tstart)
    kv("tsamp", tsamp)
    if freq_table is None:
        kv("fch1", fch1)
        kv("foff", foff)
        kv("nchans", nchans)
    else:
        out.append(_s("FREQUENCY_START"))
        for f in freq_table:
            out.append(_s("fchannel"))
            out.append(struct.pack("<d", float(f)))
        out.append(_s("FREQUENCY_END"))
    kv("nbits", nbits)
    kv("nifs", 1)
    for key, val in extra:
        if isinstance(val, str):
            out.append(_s(key))
            out.append(_s(val))
        else:
            kv(key, val)
    out.append(_s("HEADER_END"))
    with open(path, "wb") as fh:
        fh.write(b"".join(out))
        fh.write(data.tobytes())
