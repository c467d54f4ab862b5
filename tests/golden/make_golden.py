"""Generates the golden fixtures in this directory from the reference's own code.

  python tests/golden/make_golden.py cpu   # reference CPU brute force (any x86-64 host)
  python tests/golden/make_golden.py gpu   # reference GPU path (needs a B200)
  python tests/golden/make_golden.py single        # single-DM spectra (any x86-64 host)
  python tests/golden/make_golden.py single_iqrm   # single-DM spectra with IQRM (needs a B200)

Both need the reference builds under oracle/_ref/ (made by `make -C oracle ref`
from the reference sources).  Each fixture is a compressed .npz holding the
seeded input, the call's parameters and what the reference returned:

  ref_cpu_*.npz   cpucal::dedispered_fil_omp (include/cpucal.hpp:75-201): the raw
                  uint64 slices (concatenated along time) and the reference build's
                  delay table, recovered by impulse probing;
  ref_gpu_sub_*   gpucal::dedisperse_spec<T> (src/core/dedispered.cu:988-1304) with
                  the RFI stages off: coarse delays, residuals and the raw sums;
  ref_gpu_rfi_*   the RFI stages of the same call (binning, IQRM window masks,
                  zero-DM, mask file; dedispered.cu:1057-1122): window bounds,
                  masks and the processed input;
  ref_single_*    cpucal::dedisperse_spec_with_dm / dedispered_fil_with_dm
                  (include/cpucal.hpp:203-483): the spectrum, its tstart/tend/band,
                  and for Header input the samples of the caller's array it zeroed.

The CPU tests check the oracle against these files, so the oracle stays pinned
to the reference where the reference tree and a GPU are absent.
"""
import argparse
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

F32 = np.float32


def _data(rng, n, nchans, nbits):
    if nbits == 8:
        x = rng.normal(128, 20, size=(n, nchans))
        hi = 255
    else:
        x = rng.normal(32768, 2000, size=(n, nchans))
        hi = 65535
    # a few bright channels and a broadband burst give IQRM and zero-DM work
    x[:, rng.choice(nchans, size=max(1, nchans // 20), replace=False)] += 0.25 * hi
    x[n // 3:n // 3 + 3, :] += 0.2 * hi
    return np.clip(np.rint(x), 0, hi).astype(np.uint8 if nbits == 8 else np.uint16)


CPU_CASES = [
    # name, nchans, N, nbits, tsamp, fch1, foff, dm_low, dm_high, dm_step, ds, t_sample
    ("u8_ds1", 32, 1500, 8, 64e-6, 1000.0, 500 / 32, 0.0, 60.0, 1.5, 1, 0.05),
    ("u8_ds2", 40, 1200, 8, 49.152e-6, 1200.0, 0.7, 0.0, 300.0, 7.0, 2, 0.03),
    ("u16_ds3", 24, 1000, 16, 1e-4, 1100.1, 1.3, 10.0, 400.0, 13.0, 3, 0.061),
]


def make_cpu(out_dir):
    if not O.ref_cpu_available():
        raise SystemExit("oracle/_ref/libref_cpu.so missing: run `make -C oracle ref_cpu`")
    for k, (name, nchans, n, nbits, tsamp, fch1, foff, lo, hi, step, ds, ts) in enumerate(CPU_CASES):
        rng = np.random.default_rng(100 + k)
        x = _data(rng, n, nchans, nbits)
        freq = O.freq_table_fil(fch1, foff, nchans)
        fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
        out = np.concatenate(O.ref_bruteforce_cpu(x, nchans, fch1, foff, tsamp, lo, hi, fs, fe,
                                                  step, ds, ts), axis=1)
        delay = O.ref_cpu_delays(nchans, n, fch1, foff, tsamp, lo, hi, fs, fe, step)
        path = os.path.join(out_dir, f"ref_cpu_{name}.npz")
        np.savez_compressed(path, data=x, nchans=nchans, tsamp=tsamp, fch1=fch1, foff=foff,
                            dm_low=lo, dm_high=hi, freq_start=fs, freq_end=fe, dm_step=step, ds=ds,
                            t_sample=ts, delay=delay.astype(np.int32), out=out)
        print(path, os.path.getsize(path))


SUB_CASES = [
    # name, nchans, N, nbits, tsamp, fch1, foff, dm_low, dm_high, dm_step, ds, sb_width
    ("u8_sb32", 96, 2048, 8, 64e-6, 1300.0, 2.0, 0.0, 120.0, 1.0, 1, 32),
    ("u8_sb16_ds2", 64, 2500, 8, 49.152e-6, 1250.0, 3.0, 2.0, 200.0, 2.5, 2, 16),
    ("u16_sb64", 130, 1600, 16, 1e-4, 1200.0, 2.1, 0.0, 300.0, 6.0, 1, 64),
]

RFI_CASES = [
    # name, nchans, N, nbits, tsamp, ds, (mode, radius_frac, nsigma, win_sec, hop_sec), zdm,
    # mask, band (fractions of the band's span)
    ("u8_std_one_window", 128, 3000, 8, 64e-6, 1, (0, 0.1, 3.0, 0.0, 0.0), True, True, (0.0, 1.0)),
    ("u8_mad_windows_ds2", 96, 4000, 8, 64e-6, 2, (1, 0.08, 2.5, 0.05, 0.03), False, False, (0.0, 1.0)),
    ("u16_std_windows", 80, 3000, 16, 1e-4, 1, (0, 0.1, 3.0, 0.1, 0.07), False, True, (0.0, 1.0)),
    ("u8_subband_zdm", 96, 2000, 8, 64e-6, 1, (0, 0.1, 3.0, 0.0, 0.0), True, True, (0.1, 0.9)),
]


class _Iq:
    def __init__(self, mode, radius_frac, nsigma, win_sec, hop_sec):
        self.mode, self.radius_frac, self.nsigma = mode, radius_frac, nsigma
        self.geofactor, self.win_sec, self.hop_sec, self.include_tail = 1.5, win_sec, hop_sec, True


def make_gpu(out_dir):
    for k, (name, nchans, n, nbits, tsamp, fch1, foff, lo, hi, step, ds, sbw) in enumerate(SUB_CASES):
        if not O.ref_gpu_available(sbw):
            raise SystemExit(f"oracle/_ref/libref_gpu_sb{sbw}.so missing")
        rng = np.random.default_rng(200 + k)
        x = _data(rng, n, nchans, nbits)
        tsamp32, fch1_32, foff32 = float(F32(tsamp)), float(F32(fch1)), float(F32(foff))
        freq = O.freq_table_header(fch1_32, foff32, nchans)
        fs, fe = float(F32(freq[0])), float(F32(freq[-1]))
        d1, r2, info = O.ref_gpu_tables(nchans, n, tsamp32, fch1_32, foff32, lo, hi, fs, fe, step,
                                        ds, sb_width=sbw)
        out = O.ref_gpu_dedisperse_spec(x, nchans, tsamp32, fch1_32, foff32, lo, hi, fs, fe, step,
                                        ds, sb_width=sbw)
        path = os.path.join(out_dir, f"ref_gpu_sub_{name}.npz")
        np.savez_compressed(path, data=x, nchans=nchans, tsamp=tsamp32, fch1=fch1_32, foff=foff32,
                            dm_low=lo, dm_high=hi, freq_start=fs, freq_end=fe, dm_step=step, ds=ds,
                            sb_width=sbw, chan_start=info["chan_start"], chan_end=info["chan_end"],
                            delay1=d1, residual2=r2, out=out.astype(np.uint32))
        print(path, os.path.getsize(path))
    for k, (name, nchans, n, nbits, tsamp, ds, iqp, zdm, use_mask, band) in enumerate(RFI_CASES):
        rng = np.random.default_rng(300 + k)
        x = _data(rng, n, nchans, nbits)
        tsamp32, fch1_32, foff32 = float(F32(tsamp)), float(F32(1200.0)), float(F32(300.0 / nchans))
        freq = O.freq_table_header(fch1_32, foff32, nchans)
        span = freq[-1] - freq[0]
        fs = float(F32(freq[0] + band[0] * span))
        fe = float(F32(freq[0] + band[1] * span))
        bad = sorted(int(c) for c in rng.choice(nchans, size=5, replace=False))
        with tempfile.TemporaryDirectory() as td:
            mask_file = os.path.join(td, "mask.txt")
            with open(mask_file, "w") as fh:
                fh.write(" ".join(map(str, bad)) + "\n")
            iq = _Iq(*iqp)
            proc, t0, t1, masks = O.ref_gpu_rfi(x, nchans, tsamp32, fch1_32, foff32, fs, fe, ds,
                                                mask_file=mask_file, use_mask=use_mask,
                                                use_zero_dm=zdm, use_iqrm=True, iq=iq)
        path = os.path.join(out_dir, f"ref_gpu_rfi_{name}.npz")
        np.savez_compressed(path, data=x, nchans=nchans, tsamp=tsamp32, fch1=fch1_32, foff=foff32,
                            freq_start=fs, freq_end=fe, ds=ds, iq=np.array(iqp, np.float64),
                            use_zero_dm=zdm, use_mask=use_mask, bad=np.array(bad, np.int32),
                            win_t0=t0, win_t1=t1, masks=masks, processed=proc)
        print(path, os.path.getsize(path))


SINGLE_CASES = [
    # name, fil, nbits, nchans, N, tsamp, fch1, foff, tstart, tend, dm, band fractions,
    # mask, IQRM (mode, radius_frac, nsigma, win_sec, hop_sec) or None
    ("hdr_u8", False, 8, 32, 1500, 64e-6, 1200.0, 9.375, 0.02, 0.07, 30.0, (0.1, 0.9), False, None),
    ("hdr_u16_mask", False, 16, 24, 1500, 1e-4, 1100.0, 6.0, 0.02, 0.09, 25.0, (0.0, 1.0), True,
     None),
    ("fil_u32", True, 32, 16, 1000, 49.152e-6, 1300.0, 8.5, 0.01, 0.035, 20.0, (0.2, 0.8), False,
     None),
    ("fil_u8_desc_mask", True, 8, 40, 1500, 64e-6, 1500.0, -7.0, 0.0, 0.06, 40.0, (0.0, 1.0), True,
     None),
    ("hdr_u8_iqrm", False, 8, 64, 2500, 64e-6, 1200.0, 4.6875, 0.03, 0.1, 40.0, (0.0, 1.0), True,
     (0, 0.1, 3.0, 0.03, 0.02)),
    ("fil_u16_iqrm", True, 16, 48, 2000, 1e-4, 1150.0, 6.25, 0.02, 0.12, 50.0, (0.1, 0.95), False,
     (1, 0.08, 2.5, 0.0, 0.0)),
]


def make_single(out_dir, iqrm):
    """cpucal::dedisperse_spec_with_dm / dedispered_fil_with_dm (include/cpucal.hpp:203-483).
    The IQRM cases run the reference's GPU IQRM and need a B200 (iqrm=True)."""
    sys.path.insert(0, os.path.dirname(HERE))
    from sigproc_writer import write_fil
    if not O.ref_gpu_available(32):
        raise SystemExit("oracle/_ref/libref_gpu_sb32.so missing")
    for k, (name, fil, nbits, nchans, n, tsamp, fch1, foff, ts, te, dm, band, use_mask,
            iqp) in enumerate(SINGLE_CASES):
        if (iqp is not None) != iqrm:
            continue
        rng = np.random.default_rng(400 + k)
        if nbits == 32:
            x = rng.integers(0, 1 << 20, size=(n, nchans)).astype(np.uint32)
        else:
            x = _data(rng, n, nchans, nbits)
        lo_f, hi_f = (fch1, fch1 + (nchans - 1) * foff) if foff > 0 else \
            (fch1 + (nchans - 1) * foff, fch1)
        fs = float(F32(lo_f + band[0] * (hi_f - lo_f)))
        fe = float(F32(lo_f + band[1] * (hi_f - lo_f)))
        bad = sorted(int(c) for c in rng.choice(nchans, size=4, replace=False))
        iq = _Iq(*iqp) if iqp is not None else None
        with tempfile.TemporaryDirectory() as td:
            mask_file = os.path.join(td, "mask.txt")
            with open(mask_file, "w") as fh:
                fh.write(" ".join(map(str, bad)) + "\n")
            if fil:
                path = os.path.join(td, "a.fil")
                write_fil(path, x, tsamp, fch1, foff)
                spec, meta = O.ref_gpu_fil_with_dm(path, nbits, ts, te, dm, fs, fe, mask_file,
                                                   use_mask=use_mask, use_iqrm=iqp is not None,
                                                   iq=iq)
                after = None
            else:
                tsamp, fch1, foff = float(F32(tsamp)), float(F32(fch1)), float(F32(foff))
                spec, meta, after = O.ref_gpu_spec_with_dm(x, nchans, tsamp, fch1, foff, ts, te, dm,
                                                           fs, fe, mask_file, use_mask=use_mask,
                                                           use_iqrm=iqp is not None, iq=iq)
        path = os.path.join(out_dir, f"ref_single_{name}.npz")
        # the caller's array after the call, as the flat indices the reference zeroed
        extra = {} if after is None else {
            "zeroed": np.flatnonzero(after.reshape(-1) != x.reshape(-1)).astype(np.int32)}
        np.savez_compressed(path, data=x, fil=fil, nchans=nchans, tsamp=tsamp, fch1=fch1, foff=foff,
                            tstart=ts, tend=te, dm=dm, freq_start=fs, freq_end=fe,
                            use_mask=use_mask, bad=np.array(bad, np.int32),
                            iq=np.array(iqp if iqp is not None else (), np.float64),
                            spec=spec, meta=np.array(meta, np.float32), **extra)
        print(path, os.path.getsize(path))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("which", choices=["cpu", "gpu", "single", "single_iqrm"])
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.which.startswith("single"):
        make_single(a.out, a.which == "single_iqrm")
    else:
        (make_cpu if a.which == "cpu" else make_gpu)(a.out)


if __name__ == "__main__":
    main()
