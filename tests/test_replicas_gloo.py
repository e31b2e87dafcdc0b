"""Two-rank (gloo, CPU) test of the replica path used by bench.py --gpus N:
every rank projects its own replica with no grid exchange, the timing is the
max over ranks, and the throughput counts all ranks' solves."""
import json
import os
import socket
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import json, os, sys, time
    sys.path.insert(0, {root!r})
    sys.path.insert(0, os.path.join({root!r}, "tests"))
    from mydemcfd_b200 import replicas, workloads as W
    from oracle import oracle as O
    from _cases import ref_grid
    r = replicas.init(replicas.from_env(), "gloo", timeout_s=60)
    O.set_num_threads(1)
    case = W.plain_case(24, seed=7 + r.rank)          # each rank its own replica
    replicas.barrier(r)
    t0 = time.perf_counter()
    pd, _, st = O.solve(ref_grid(case), tol=1e-9, stop_rule=O.STOP_REL_TRUE)
    ms = (time.perf_counter() - t0) * 1e3 + 50.0 * r.rank   # rank 1 made artificially slower
    replicas.barrier(r)
    ms_max = replicas.max_over_ranks(r, ms)
    out = dict(rank=r.rank, world=r.world, ms=ms, ms_max=ms_max, iters=st["iterations"],
               value=replicas.throughput(r, 1, ms_max), conv=st["converged"])
    print("RESULT " + json.dumps(out), flush=True)
    replicas.finish(r)
""")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_replicas(tmp_path, oracle_lib):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), OMP_NUM_THREADS="1", CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            p.kill()
            pytest.fail("rank did not finish")
        assert p.returncode == 0, o
        outs.append(json.loads([l for l in o.splitlines() if l.startswith("RESULT ")][0][7:]))
    r0, r1 = sorted(outs, key=lambda d: d["rank"])
    assert r0["world"] == r1["world"] == 2
    assert r0["conv"] and r1["conv"]
    # both ranks agree on the slowest rank's time, which is rank 1's
    assert r0["ms_max"] == r1["ms_max"] == pytest.approx(max(r0["ms"], r1["ms"]))
    assert r0["ms_max"] >= r1["ms"] - 1e-9
    # whole-job throughput: 2 solves in the slowest rank's time
    assert r0["value"] == pytest.approx(2 / (r0["ms_max"] / 1e3))
