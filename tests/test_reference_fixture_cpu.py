"""Real data: the reference's own test file, tests/FRB180417.fil of the reference
tree (336 channels of 8-bit samples, 5120 samples of 1.266 ms, the burst FRB
180417 at DM 474.8, docs/quick_start.md:65).  It is read where the reference tree
is ($ASTROFLOW_REFERENCE, else the tree oracle/_ref was built from); elsewhere
these tests skip.
They pin on real data: the library's SIGPROC header reader against the drop-in's
host reader, the oracle's brute force and single-DM spectrum against the
reference's own builds, the reference's DM-0 identity
(python/tests/test_dedispered.py:20-57) and the published DM of the burst."""
import os

import numpy as np
import pytest

from oracle import oracle as O

REFERENCE_TREE = O.reference_tree()
FIL = os.path.join(REFERENCE_TREE, "tests", "FRB180417.fil")
F32 = np.float32

pytestmark = pytest.mark.skipif(not os.path.exists(FIL), reason="reference tree absent")


@pytest.fixture(scope="module")
def fil():
    from astroflow_b200 import _astroflow_core as C

    fb = C.Filterbank(FIL)
    x = np.ascontiguousarray(fb.data.reshape(fb.ndata, fb.nchans))
    return fb, x


def test_header_readers_agree(fil):
    """dd_fil_read_header (the library, host code) and the drop-in's host reader give
    the same header and the same ascending frequency table."""
    from astroflow_b200 import ingest

    fb, x = fil
    fh, table = ingest.fil_header(FIL)
    assert (fh["nchans"], fh["nbits"], fh["ndata"], fh["nifs"]) == (fb.nchans, fb.nbits, fb.ndata, 1)
    assert (fh["tsamp"], fh["fch1"], fh["foff"]) == (fb.tsamp, fb.fch1, fb.foff)
    assert x.shape == (5120, 336) and x.dtype == np.uint8
    np.testing.assert_array_equal(table, O.freq_table_fil(fb.fch1, fb.foff, fb.nchans))


@pytest.mark.skipif(not O.ref_gpu_available(32), reason="reference build absent")
def test_dm0_window_is_the_raw_data(fil):
    """The reference's own known answer: at DM 0 the spectrum of [0, 0.5) s over the
    whole band is the raw data (its test checks the same identity against an
    independent reader); the reference build and the oracle agree."""
    fb, x = fil
    top = fb.fch1 + (fb.nchans - 1) * fb.foff
    ref, meta = O.ref_gpu_fil_with_dm(FIL, 8, 0.0, 0.5, 0.0, fb.fch1, top)
    ntimes = int((0.5 - 0.0) / fb.tsamp)
    assert ref.shape == (ntimes, fb.nchans)
    np.testing.assert_array_equal(ref, x[:ntimes])
    g = O.single_dm_geometry(fb.nchans, fb.ndata, fb.tsamp, fb.fch1, fb.foff, 0.0, 0.5, 0.0,
                             fb.fch1, top, fil=True)
    np.testing.assert_array_equal(O.single_dm_spectrum(x, fb.nchans, g), ref)


@pytest.mark.skipif(not O.ref_gpu_available(32), reason="reference build absent")
@pytest.mark.parametrize("window,band", [((1.5, 2.5), (1130.0, 1465.0)),
                                         ((1.9, 2.3), (1200.5, 1400.0)),
                                         ((0.0, 6.0), (1130.0, 1465.0))])
def test_oracle_spectrum_matches_reference_at_the_burst_dm(fil, window, band):
    fb, x = fil
    ref, meta = O.ref_gpu_fil_with_dm(FIL, 8, window[0], window[1], 474.8, *band)
    g = O.single_dm_geometry(fb.nchans, fb.ndata, fb.tsamp, fb.fch1, fb.foff, window[0],
                             window[1], 474.8, *band, fil=True)
    np.testing.assert_array_equal(O.single_dm_spectrum(x, fb.nchans, g), ref)
    assert (F32(window[0]), F32(g.tend), F32(g.freq_start), F32(g.freq_end)) == tuple(meta)


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
def test_brute_force_oracle_matches_reference_build(fil):
    """DM 10-600 step 1 (the quick start's search grid) over the whole band: the
    oracle with the reference build's own delay table equals the reference's
    cpucal::dedispered_fil_omp sample for sample."""
    fb, x = fil
    args = (fb.tsamp, 10.0, 600.0, 1130.0, 1465.0, 1.0)
    ref = O.ref_bruteforce_cpu(x, fb.nchans, fb.fch1, fb.foff, *args[:5], args[5], 1, 6.0)
    delay = O.ref_cpu_delays(fb.nchans, fb.ndata, fb.fch1, fb.foff, *args)
    freq = O.freq_table_fil(fb.fch1, fb.foff, fb.nchans)
    got = O.bruteforce_cpu(x, fb.nchans, freq, *args[:5], args[5], 1, 6.0, delay=delay)
    assert len(got) == len(ref) == 2
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)


def test_burst_found_at_the_published_dm(fil):
    """The oracle's brute force over DM 10-600 finds the burst at 474.8 +- 3: the
    DM row whose detrended series has the highest peak over its spread, at 2.03 s."""
    fb, x = fil
    freq = O.freq_table_fil(fb.fch1, fb.foff, fb.nchans)
    raw = O.bruteforce_cpu(x, fb.nchans, freq, fb.tsamp, 10.0, 600.0, 1130.0, 1465.0, 1.0, 1,
                           6.0)[0].astype(np.float64)
    k = 64
    trend = np.array([np.convolve(r, np.ones(k) / k, mode="same") for r in raw])
    d = (raw - trend)[:, k:-k]
    box = np.array([np.convolve(r, np.ones(2), mode="valid") for r in d])
    snr = box.max(axis=1) / box.std(axis=1)
    best = int(np.argmax(snr))
    assert abs(10.0 + best - 474.8) <= 3.0, (10 + best, snr[best])
    assert snr[best] > 10.0
    t_peak = (int(np.argmax(box[best])) + k) * fb.tsamp
    assert abs(t_peak - 2.03) < 0.05, t_peak
