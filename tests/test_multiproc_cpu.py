"""Replicas across ranks on CPU (gloo, world size 2): every rank runs the same
collective steps, the job's time is the slowest rank's, the job's throughput
sums all ranks' units, each rank gets its own chunk, and a rank that fails
before a collective makes the others' next collective end with an error
instead of waiting forever.  The per-rank "step" here is the oracle's subband
sums on the rank's chunk (the GPU kernels need a GPU)."""
import os
import socket
import subprocess
import sys
import textwrap

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(body: str, world: int = 2, timeout: float = 120.0):
    port = _free_port()
    script = textwrap.dedent(body)
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), PYTHONPATH=REPO,
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", script], env=env, cwd=REPO,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            o, e = p.communicate()
        outs.append((p.returncode, o, e))
    return outs


def test_replicas_timing_and_job_rate():
    outs = _run_ranks("""
        import json
        import numpy as np
        from astroflow_b200.replicas import Replicas
        from astroflow_b200.synth import ChunkSpec, make_chunk
        from oracle import oracle as O

        rep = Replicas("gloo", timeout_s=60)
        spec = ChunkSpec(nchans=64, nsamp=1024, nbits=8, seed=rep.chunk_seed(1234))
        x, hdr = make_chunk(spec)
        freq = O.freq_table_header(hdr["fch1"], hdr["foff"], 64)
        fs, fe = float(np.float32(freq[0])), float(np.float32(freq[-1]))
        plan = O.subband_plan(freq, 1024, 0.0, 50.0, fs, fe, 1.0, 1, sb_width=16)
        d1 = np.zeros((plan.ndm_nom, plan.chan_end - plan.chan_start + 1), np.int32)
        r2 = np.zeros((plan.dm_steps, plan.nsb), np.int32)
        rep.barrier()
        out = O.subband_sums(x, 64, plan, d1, r2)
        rep.barrier()
        units = out.shape[0] * out.shape[1]
        secs = 1.0 + rep.rank          # stand-in step times: rank 1 is the slowest
        rate = rep.job_rate(units, secs)
        slowest = rep.max(secs)
        print(json.dumps({"rank": rep.rank, "world": rep.world, "units": units, "rate": rate,
                          "slowest": slowest, "checksum": int(out.sum()),
                          "dm0_equals_band_sum": bool((out[0] == x[:, plan.chan_start:plan.chan_end + 1].sum(1)).all())}))
        rep.close()
    """)
    import json

    res = []
    for rc, o, e in outs:
        assert rc == 0, e
        res.append(json.loads(o.strip().splitlines()[-1]))
    assert [r["rank"] for r in res] == [0, 1] and all(r["world"] == 2 for r in res)
    units = res[0]["units"]
    for r in res:
        assert r["slowest"] == 2.0
        assert r["rate"] == pytest.approx(2 * units / 2.0)
        assert r["dm0_equals_band_sum"]
    assert res[0]["checksum"] != res[1]["checksum"], "ranks must work on their own chunks"


def test_failed_rank_ends_the_others_collective_with_an_error():
    outs = _run_ranks("""
        import sys
        from astroflow_b200.replicas import Replicas

        rep = Replicas("gloo", timeout_s=5)
        rep.barrier()
        if rep.rank == 1:
            sys.exit(3)            # leaves between steps, before the next collective
        try:
            rep.max(1.0)
        except Exception as exc:   # the collective ends with an error, no hang
            print("error:", type(exc).__name__)
            sys.exit(0)
        print("no error")
        sys.exit(1)
    """, timeout=90)
    (rc0, o0, e0), (rc1, _, _) = outs
    assert rc1 == 3
    assert rc0 == 0 and "error:" in o0, (o0, e0)


def test_single_process_needs_no_process_group():
    from astroflow_b200.replicas import Replicas

    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        rep = Replicas("gloo")
        assert (rep.world, rep.rank, rep.pg) == (1, 0, None)
        assert rep.max(2.5) == 2.5 and rep.job_rate(100, 2.0) == 50.0
        assert rep.chunk_seed(7) == 7
        rep.barrier()
        rep.close()
    finally:
        os.environ.update(env)
