"""SIGPROC headers through the library's reader (dd_fil_read_header) against the
reference-equivalent host reader of the drop-in module (src/data/filterbank.cpp:
319-452 and the channel flip of :793-842).  No GPU needed."""
import numpy as np
import pytest

from astroflow_b200 import _astroflow_core as C
from astroflow_b200 import ingest
from sigproc_writer import write_fil

CASES = [
    # nbits, nsamp, nchans, fch1, foff, table, extra
    (8, 50, 16, 1500.0, -2.0, None, ()),
    (16, 33, 8, 1100.0, 0.5, None, [("refdm", 12.5), ("ibeam", 3), ("rawdatafile", "a.raw")]),
    (32, 20, 12, 1200.0, 1.25, None, [("nsamples", 20), ("az_start", 1.0)]),
    (8, 40, 8, 0.0, 0.0, 1000.0 + np.arange(8) * 3.0, ()),
    (16, 25, 10, 1400.0, -0.75, None, [("nifs", 1), ("period", 0.5)]),
]


@pytest.mark.parametrize("case", CASES)
def test_header_matches_the_host_reader(case, tmp_path):
    nbits, n, nch, fch1, foff, table, extra = case
    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32}[nbits]
    p = str(tmp_path / "a.fil")
    write_fil(p, np.zeros((n, nch), dt), 64e-6, fch1, foff, freq_table=table, extra=extra)
    h, freq = ingest.fil_header(p)
    f = C.Filterbank(p)
    assert (h["nbits"], h["nchans"], h["nifs"], h["ndata"]) == (f.nbits, f.nchans, f.nifs, f.ndata)
    assert (h["fch1"], h["foff"], h["tsamp"], h["tstart"]) == (f.fch1, f.foff, f.tsamp, f.tstart)
    assert h["header_bytes"] == f.header_size
    assert h["flipped"] == int(foff < 0 and table is None)
    np.testing.assert_array_equal(freq, f.frequency_table)


def test_partial_last_sample_is_dropped(tmp_path):
    p = str(tmp_path / "a.fil")
    write_fil(p, np.zeros((10, 8), np.uint8), 1e-4, 1000.0, 1.0)
    with open(p, "ab") as fh:
        fh.write(b"\x01\x02\x03")
    assert ingest.fil_header(p)[0]["ndata"] == 10 == C.Filterbank(p).ndata


def test_header_errors(tmp_path):
    p = str(tmp_path / "bad.fil")
    write_fil(p, np.zeros((4, 4), np.uint8), 1e-4, 1100.0, 0.5, extra=[("not_a_key", 1)])
    with pytest.raises(ValueError, match="unknown parameter : not_a_key"):
        ingest.fil_header(p)
    q = str(tmp_path / "junk.fil")
    with open(q, "wb") as fh:
        fh.write(b"\x05\x00\x00\x00hello" + bytes(64))
    with pytest.raises(ValueError, match="Non-Standard file format"):
        ingest.fil_header(q)
    r = str(tmp_path / "nifs2.fil")
    write_fil(r, np.zeros((4, 8), np.uint8), 1e-4, 1100.0, -0.5, extra=[("nifs", 2)])
    with pytest.raises(ValueError, match="nifs == 1"):
        ingest.fil_header(r)
    with pytest.raises(ValueError, match="cannot open"):
        ingest.fil_header(str(tmp_path / "missing.fil"))
