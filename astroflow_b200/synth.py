"""Seeded synthetic filterbank chunks with the shapes of astroflow's workloads.

Data are time-major [nsamp, nchans] in ascending frequency order (the order the
reference's readers produce after flipping foff < 0 files, src/data/filterbank.cpp:793-842):
Gaussian noise rounded and clipped to the sample type, dispersed Gaussian
pulses with delays 4148.808*DM*(f^-2 - f_hi^-2) s rounded at injection
(python/astroflow/dataset/simulator.py:22, 122-124), optional sinusoidal RFI
channels and broadband zero-DM impulses.  Small chunks are generated with
numpy; large ones on a CUDA device with torch (same statistics, seeded).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

KDM = 4148.808


@dataclass
class ChunkSpec:
    nchans: int = 1024
    nsamp: int = 1 << 17
    nbits: int = 8
    f_hi: float = 1500.0          # MHz, top of the band
    bandwidth: float = 500.0      # MHz
    tsamp: float = 49.152e-6      # s
    seed: int = 0
    mean: Optional[float] = None  # default 128 (8-bit) / 32768 (16-bit) / 1e6 (32-bit)
    sigma: Optional[float] = None # default 20 / 2000 / 6e4
    pulses: Sequence[Tuple[float, float, float, float]] = ()  # (dm, t0 s, width s, amplitude)
    rfi_frac: float = 0.0         # fraction of channels with a sinusoid
    rfi_amp: float = 60.0
    rfi_period: Tuple[int, int] = (2, 200)
    impulses: int = 0             # broadband zero-DM impulses
    imp_amp: float = 50.0
    imp_width: Tuple[int, int] = (1, 4)

    @property
    def foff(self) -> float:
        return self.bandwidth / self.nchans

    @property
    def fch1(self) -> float:
        """Lowest channel frequency (ascending order)."""
        return self.f_hi - (self.nchans - 1) * self.foff

    def header(self) -> dict:
        return dict(mjd=0.0, tsamp=self.tsamp, fch1=self.fch1, foff=self.foff, nbits=self.nbits,
                    nchans=self.nchans, ndata=self.nsamp, filename="synthetic")

    def freqs(self) -> np.ndarray:
        return self.fch1 + np.arange(self.nchans) * self.foff


def _defaults(spec: ChunkSpec):
    if spec.nbits == 8:
        return (128.0 if spec.mean is None else spec.mean, 20.0 if spec.sigma is None else spec.sigma, 255)
    if spec.nbits == 32:
        # float32 holds every integer below 2^24 exactly
        return (1e6 if spec.mean is None else spec.mean, 6e4 if spec.sigma is None else spec.sigma,
                float(2 ** 32 - 1))
    return (32768.0 if spec.mean is None else spec.mean, 2000.0 if spec.sigma is None else spec.sigma, 65535)


def _extras(spec: ChunkSpec, rng: np.random.Generator):
    """Additive signal: ("add", rows, cols, values) pulses, ("sin", channel, (period,
    phase)) RFI channels and ("imp", start, width) broadband impulses."""
    f = spec.freqs()
    adds: list = []
    for dm, t0, width, amp in spec.pulses:
        delay = KDM * dm * (f ** -2 - spec.f_hi ** -2)
        w = max(width / spec.tsamp, 0.5)
        half = int(math.ceil(4 * w))
        offs = np.arange(-half, half + 1)
        prof = amp * np.exp(-0.5 * (offs / w) ** 2)
        for c in range(spec.nchans):
            centre = int(np.rint((t0 + delay[c]) / spec.tsamp))
            rows = centre + offs
            ok = (rows >= 0) & (rows < spec.nsamp)
            if ok.any():
                adds.append(("add", rows[ok], np.full(int(ok.sum()), c), prof[ok]))
    if spec.rfi_frac > 0:
        nr = max(1, int(round(spec.rfi_frac * spec.nchans)))
        chans = rng.choice(spec.nchans, size=nr, replace=False)
        periods = rng.integers(spec.rfi_period[0], spec.rfi_period[1] + 1, size=nr)
        phases = rng.uniform(0, 2 * np.pi, size=nr)
        for c, p, ph in zip(chans, periods, phases):
            adds.append(("sin", int(c), (float(p), float(ph))))
    for _ in range(spec.impulses):
        t = int(rng.integers(0, spec.nsamp))
        wd = int(rng.integers(spec.imp_width[0], spec.imp_width[1] + 1))
        adds.append(("imp", t, wd))
    return adds


def make_chunk(spec: ChunkSpec) -> Tuple[np.ndarray, dict]:
    """Host (numpy) chunk [nsamp, nchans] of uint8/uint16/uint32 and its header."""
    rng = np.random.default_rng(spec.seed)
    mean, sigma, vmax = _defaults(spec)
    x = rng.normal(mean, sigma, size=(spec.nsamp, spec.nchans)).astype(np.float32)
    for item in _extras(spec, rng):
        if item[0] == "sin":
            _, c, (p, ph) = item
            t = np.arange(spec.nsamp, dtype=np.float32)
            x[:, c] += spec.rfi_amp * np.sin(2 * np.pi * t / p + ph)
        elif item[0] == "imp":
            _, t, wd = item
            x[t:t + wd, :] += spec.imp_amp
        else:
            _, rows, cols, vals = item
            np.add.at(x, (rows, cols), vals)
    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32}[spec.nbits]
    if spec.nbits == 32:
        return np.clip(np.rint(x.astype(np.float64)), 0, vmax).astype(dt), spec.header()
    return np.clip(np.rint(x), 0, vmax).astype(dt), spec.header()


def make_chunk_device(spec: ChunkSpec, device: int = 0):
    """Device (torch) chunk with the same construction, generated on the GPU."""
    import torch

    if spec.nbits not in (8, 16):
        raise ValueError("device chunks are generated for 8- and 16-bit samples")
    mean, sigma, vmax = _defaults(spec)
    rng = np.random.default_rng(spec.seed)
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(spec.seed)
    dt = torch.uint8 if spec.nbits == 8 else torch.uint16
    out = torch.empty((spec.nsamp, spec.nchans), dtype=dt, device=f"cuda:{device}")
    rows_per = max(1, (1 << 27) // spec.nchans)
    extras = _extras(spec, rng)
    for r0 in range(0, spec.nsamp, rows_per):
        r1 = min(spec.nsamp, r0 + rows_per)
        blk = torch.randn((r1 - r0, spec.nchans), generator=g, device=out.device) * sigma + mean
        for item in extras:
            if item[0] == "sin":
                _, c, (p, ph) = item
                t = torch.arange(r0, r1, device=out.device, dtype=torch.float32)
                blk[:, c] += spec.rfi_amp * torch.sin(2 * math.pi * t / p + ph)
            elif item[0] == "imp":
                _, t, wd = item
                a, b = max(t, r0), min(t + wd, r1)
                if a < b:
                    blk[a - r0:b - r0, :] += spec.imp_amp
            else:
                _, rows, cols, vals = item
                sel = (rows >= r0) & (rows < r1)
                if sel.any():
                    rr = torch.as_tensor(rows[sel] - r0, device=out.device)
                    cc = torch.as_tensor(cols[sel], device=out.device)
                    vv = torch.as_tensor(vals[sel], device=out.device, dtype=torch.float32)
                    blk.index_put_((rr, cc), vv, accumulate=True)
        out[r0:r1] = torch.clamp(torch.round(blk), 0, vmax).to(torch.int32).to(dt)
    return out, spec.header()


# ---------------------------------------------------------------- heterogeneous batches
@dataclass
class BatchChunk:
    """One chunk of a heterogeneous batch and its dedispersion plan."""
    spec: ChunkSpec
    dm_high: float
    dm_step: float
    time_downsample: int
    subband_width: int


def draw_batch(n: int = 64, seed: int = 2024, subband_width: int = 32,
               log2_nsamp: Tuple[float, float] = (15.0, 19.0)) -> List[BatchChunk]:
    """Seeded draw of a heterogeneous batch: nchan in {1024, 2048, 4096}, 8- or 16-bit
    samples, nsamp log-uniform in [2^15, 2^19] (log2_nsamp), band 1000-1500 or
    1250-1550 MHz, maximum DM in {500, 1500, 3000} with a step in {0.5, 1, 1.5, 2},
    time downsampling in {1, 2, 4, 8}, one dispersed pulse per chunk at a random DM."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nchans = int(rng.choice([1024, 2048, 4096]))
        nbits = int(rng.choice([8, 16]))
        nsamp = int(round(2 ** rng.uniform(*log2_nsamp)))
        f_hi, bw = ((1500.0, 500.0), (1550.0, 300.0))[int(rng.integers(2))]
        dm_high = float(rng.choice([500.0, 1500.0, 3000.0]))
        dm_step = float(rng.choice([0.5, 1.0, 1.5, 2.0]))
        ds = int(rng.choice([1, 2, 4, 8]))
        tsamp = 49.152e-6
        dm = float(rng.uniform(0.1, 0.9) * dm_high)
        amp = 12.0 if nbits == 8 else 1200.0
        spec = ChunkSpec(nchans=nchans, nsamp=nsamp, nbits=nbits, f_hi=f_hi, bandwidth=bw,
                         tsamp=tsamp, seed=seed * 1000 + i,
                         pulses=[(dm, float(rng.uniform(0.1, 0.6)) * nsamp * tsamp, 1e-3, amp)])
        out.append(BatchChunk(spec, dm_high, dm_step, ds, subband_width))
    return out
