"""Serving loop: streaming beams and ad-hoc file requests on one GPU.

astroflow's nearest thing to serving is its directory-polling monitor mode
(python/astroflow/search.py:868-993), which dedisperses one file at a time.
Here requests are served with continuous batching:

  * beams: each beam is a dd_stream (its max-delay tail stays on the device) fed
    one chunk at a time; a chunk's result is the first chunk/ds columns of the
    plain call on [tail | chunk] (see dd_stream_open);
  * files: ad-hoc requests dedispersed by a plain call on the whole file.

Requests that arrive while others are on the GPU are admitted as CUDA-stream
slots and HBM budget free up: beams reserve their memory when opened, files
when admitted (first come, first served).  Every admitted request runs on its
own CUDA stream, so copies and kernels of different requests overlap on the
device.  Plans of files are built and released on a worker thread so the loop
keeps launching beam chunks meanwhile.  Latency is arrival -> result ready
(beam chunks: DM-time rows copied to pinned host memory; files: DM-time rows in
device memory), measured on the host.
"""
from __future__ import annotations

import collections
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import numpy as np

from .dedisp import Plan, Stream


def _torch():
    import torch
    return torch


@dataclass
class Ticket:
    """One request: a beam chunk or a file."""
    id: int
    kind: str                       # "chunk" or "file"
    arrival: float                  # host monotonic time
    units: int = 0                  # DM-trial x output samples
    launched: Optional[float] = None
    done: Optional[float] = None
    result: Any = None              # chunk: host numpy view; file: device tensor
    error: Optional[str] = None
    beam: Any = None
    payload: Any = None
    event: Any = None
    slot: int = -1                  # file: CUDA-stream slot
    reserved_bytes: int = 0         # file: HBM reserved while admitted

    @property
    def latency(self) -> Optional[float]:
        return None if self.done is None else self.done - self.arrival


@dataclass
class Beam:
    name: str
    stream: Stream
    cuda_stream: Any
    chunk_dev: Any
    outs: List[Any]                 # device outputs (ring)
    host_outs: List[Any]            # pinned host outputs (ring)
    reserved: int
    pending: collections.deque = field(default_factory=collections.deque)
    inflight: Optional[Ticket] = None
    slot: int = 0


class Server:
    """Continuous-batching dedispersion server on one GPU.

    hbm_budget_gb bounds the device memory of admitted requests (beams from
    open_beam on, files while they run); file_slots bounds files in flight."""

    def __init__(self, device: int = 0, hbm_budget_gb: float = 150.0, file_slots: int = 4,
                 ring: int = 3, keep_file_results: bool = False):
        torch = _torch()
        from . import _lib
        _lib.load()
        self.device = device
        self.budget = int(hbm_budget_gb * 1e9)
        self.reserved = 0
        self.ring = ring
        self.keep_file_results = keep_file_results
        self.beams: Dict[str, Beam] = {}
        self.files: collections.deque = collections.deque()   # waiting for admission
        self.file_streams = [torch.cuda.Stream(device) for _ in range(file_slots)]
        self.free_file_streams = list(range(file_slots))
        self.files_building: Dict[int, Ticket] = {}
        self.files_running: List[Ticket] = []
        self.finished: List[Ticket] = []
        self.files_released = 0
        self._ids = 0
        self._jobs: "queue.Queue" = queue.Queue()
        self._built: "queue.Queue" = queue.Queue()
        self._released: "queue.Queue" = queue.Queue()
        self._worker = threading.Thread(target=self._work, daemon=True)
        self._worker.start()

    # ------------------------------------------------------------------ requests
    def _next_id(self) -> int:
        self._ids += 1
        return self._ids

    def open_beam(self, name: str, header, dm_low: float, dm_high: float, freq_start: float,
                  freq_end: float, dm_step: float = 1.0, **kwargs) -> Beam:
        """Open a beam; header describes one chunk (ndata = samples per chunk)."""
        torch = _torch()
        torch.cuda.set_device(self.device)
        st = Stream(header, dm_low, dm_high, freq_start, freq_end, dm_step, device=self.device,
                    **kwargs)
        out_bytes = st.out_shape[0] * st.out_shape[1] * 4
        need = int(st.info["workspace_bytes"]) + self.ring * out_bytes + \
            st.chunk_shape[0] * st.chunk_shape[1] * st.nbits // 8
        if self.reserved + need > self.budget:
            st.close()
            raise MemoryError(f"beam {name} needs {need / 1e9:.2f} GB beyond the HBM budget")
        dt = {8: torch.uint8, 16: torch.uint16}[st.nbits]
        b = Beam(name=name, stream=st, cuda_stream=torch.cuda.Stream(self.device),
                 chunk_dev=torch.empty(st.chunk_shape, dtype=dt, device=f"cuda:{self.device}"),
                 outs=[st.empty_output() for _ in range(self.ring)],
                 host_outs=[torch.empty(st.out_shape, dtype=torch.int32, pin_memory=True)
                            for _ in range(self.ring)],
                 reserved=need)
        self.reserved += need
        self.beams[name] = b
        return b

    def close_beam(self, name: str) -> None:
        b = self.beams.pop(name)
        b.cuda_stream.synchronize()
        self.reserved -= b.reserved
        b.stream.close()

    def submit_chunk(self, beam: Beam, host_chunk, arrival: Optional[float] = None) -> Ticket:
        """host_chunk: pinned host tensor of the beam's chunk shape (kept until launched)."""
        t = Ticket(self._next_id(), "chunk", time.monotonic() if arrival is None else arrival,
                   units=beam.stream.out_shape[0] * beam.stream.out_shape[1], beam=beam,
                   payload=host_chunk)
        beam.pending.append(t)
        return t

    def submit_file(self, host_data, header, plan_kwargs: dict,
                    arrival: Optional[float] = None) -> Ticket:
        """host_data: pinned host tensor [ndata, nchans]; plan_kwargs: Plan arguments
        after the header (dm_low, dm_high, freq_start, freq_end, ...)."""
        t = Ticket(self._next_id(), "file", time.monotonic() if arrival is None else arrival,
                   payload=(host_data, header, plan_kwargs))
        self.files.append(t)
        return t

    # ------------------------------------------------------------------ worker
    def _work(self):
        torch = _torch()
        torch.cuda.set_device(self.device)
        while True:
            job = self._jobs.get()
            if job is None:
                return
            kind, t = job
            try:
                if kind == "build":
                    host, header, kw = t.payload
                    try:
                        plan = Plan(header, device=self.device, **kw)
                    except MemoryError:
                        # torch's caching allocator may hold the free memory the plan
                        # needs (the plan allocates from the stream-ordered pool):
                        # release its unused blocks and build once more
                        torch.cuda.synchronize(self.device)
                        torch.cuda.empty_cache()
                        plan = Plan(header, device=self.device, **kw)
                    t.payload = (host, header, kw, plan)
                    self._built.put(t)
                else:  # release, stream-ordered on the file's stream (its work is done)
                    plan = t.payload[3]
                    plan.close(stream=self.file_streams[t.slot])
                    self._released.put(t)
            except Exception as exc:  # reported on the ticket
                t.error = f"{type(exc).__name__}: {exc}"
                if kind == "build":
                    self._built.put(t)

    # ------------------------------------------------------------------ loop
    def _file_need(self, t: Ticket) -> int:
        host, header, kw = t.payload[:3]
        g = (lambda k: header[k]) if isinstance(header, dict) else (lambda k: getattr(header, k))
        n, c, bits = int(g("ndata")), int(g("nchans")), int(g("nbits"))
        # input, prepared copy, output rows (an upper bound on DM trials), one
        # time tile of subband sums (the library's default budget: 2 GiB)
        lo, hi, step = kw["dm_low"], kw["dm_high"], kw.get("dm_step", 1.0)
        ndm = int((hi - lo) / step) + 1
        return 2 * n * c * bits // 8 + ndm * n * 4 + (2 << 30)

    def step(self) -> bool:
        """One pass: finish completed work, launch ready beam chunks, admit files.
        Returns True if anything is still queued or running."""
        torch = _torch()
        now = time.monotonic
        # completions
        for b in self.beams.values():
            t = b.inflight
            if t is not None and t.event.query():
                t.done = now()
                b.inflight = None
                self.finished.append(t)
        for t in list(self.files_running):
            if t.event.query():
                t.done = now()
                self.files_running.remove(t)
                self.finished.append(t)
                if not self.keep_file_results:
                    t.result = None
                t.payload[0] = None  # the device copy of the input
                self._jobs.put(("release", t))
        # files whose plans the worker has released give back their slot and memory
        while True:
            try:
                t = self._released.get_nowait()
            except queue.Empty:
                break
            self.free_file_streams.append(t.slot)
            self.reserved -= t.reserved_bytes
            self.files_released += 1
        # beam chunks: one in flight per beam, in order
        for b in self.beams.values():
            if b.inflight is None and b.pending:
                t = b.pending.popleft()
                s = b.cuda_stream
                with torch.cuda.stream(s):
                    b.chunk_dev.copy_(t.payload, non_blocking=True)
                    out = b.outs[b.slot]
                    b.stream.push(b.chunk_dev, out, s)
                    host = b.host_outs[b.slot]
                    host.copy_(out.view(torch.int32), non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(s)
                t.event, t.launched, t.payload = ev, now(), None
                t.result = host.numpy().view(np.uint32)
                b.slot = (b.slot + 1) % self.ring
                b.inflight = t
        # files: plans built by the worker start running
        while True:
            try:
                t = self._built.get_nowait()
            except queue.Empty:
                break
            self.files_building.pop(t.id, None)
            if t.error:
                t.done = now()
                self.finished.append(t)
                self.free_file_streams.append(t.slot)
                self.reserved -= t.reserved_bytes
                continue
            host, header, kw, plan = t.payload
            s = self.file_streams[t.slot]
            with torch.cuda.stream(s):
                dt = {8: torch.uint8, 16: torch.uint16}[plan.nbits]
                x = torch.empty(tuple(host.shape), dtype=dt, device=f"cuda:{self.device}")
                x.copy_(host, non_blocking=True)
                out = plan.empty_output()
                plan.run(x, out, s)
                ev = torch.cuda.Event()
                ev.record(s)
            t.units = plan.out_shape[0] * plan.out_shape[1]
            t.event, t.launched, t.result = ev, now(), out
            t.payload = [x, header, kw, plan]
            self.files_running.append(t)
        # admission of files (first come, first served)
        while self.files and self.free_file_streams:
            t = self.files[0]
            need = self._file_need(t)
            if self.reserved + need > self.budget and (self.files_running or self.files_building):
                break
            self.files.popleft()
            t.reserved_bytes = need
            self.reserved += need
            t.slot = self.free_file_streams.pop()
            self.files_building[t.id] = t
            self._jobs.put(("build", t))
        busy = any(b.inflight or b.pending for b in self.beams.values())
        releasing = len(self.free_file_streams) < len(self.file_streams) and not (
            self.files_building or self.files_running)
        return busy or releasing or bool(self.files or self.files_building or self.files_running)

    def drain(self, timeout: float = 600.0) -> None:
        t0 = time.monotonic()
        while self.step():
            if time.monotonic() - t0 > timeout:
                raise TimeoutError("requests still running")
            time.sleep(0.0002)

    def close(self) -> None:
        self.drain()
        for name in list(self.beams):
            self.close_beam(name)
        self._jobs.put(None)
        self._worker.join(timeout=60)

    # ------------------------------------------------------------------ report
    def stats(self, since: float = 0.0) -> dict:
        def summary(ts):
            lat = np.array([t.latency for t in ts if t.latency is not None and not t.error])
            if lat.size == 0:
                return {"n": 0}
            return {"n": int(lat.size), "p50_s": float(np.percentile(lat, 50)),
                    "p99_s": float(np.percentile(lat, 99)), "max_s": float(lat.max())}
        done = [t for t in self.finished if t.arrival >= since]
        return {"chunks": summary([t for t in done if t.kind == "chunk"]),
                "files": summary([t for t in done if t.kind == "file"]),
                "errors": [t.error for t in done if t.error],
                "units": int(sum(t.units for t in done if not t.error))}
