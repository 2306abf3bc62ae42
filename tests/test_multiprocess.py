"""The cross-rank steps of a multi-GPU run (barrier, slowest-rank timing, job
throughput, work sharding), with two ranks as separate processes on a gloo
group over 127.0.0.1 — the same code bench.py runs over NCCL with one process
per GPU. The data path itself has no collective: ranks shard rasters."""
import json
import os
import socket
import subprocess
import sys

from map_b200 import multigpu as MG

HERE = os.path.dirname(os.path.abspath(__file__))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(mode, world=2, timeout=120):
    port = _port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "_mp_worker.py"), mode], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            o, e = p.communicate()
        lines = [l for l in o.splitlines() if l.startswith("{")]
        outs.append((p.returncode, json.loads(lines[-1]) if lines else None, e[-2000:]))
    return outs


def test_two_ranks_agree_on_the_slowest_time_and_split_the_work():
    outs = _run("ok")
    res = [o[1] for o in outs]
    assert all(o[0] == 0 for o in outs), outs
    assert {r["rank"] for r in res} == {0, 1}
    assert all(r["world"] == 2 and r["slowest_ms"] == 15.0 for r in res)
    assert all(abs(r["gcells"] - 2e9 / 15e-3 / 1e9) < 1e-9 for r in res)
    a, b = sorted(res, key=lambda r: r["rank"])
    assert sorted(a["shard"] + b["shard"]) == list(range(40)) and not set(a["shard"]) & set(b["shard"])
    assert abs(a["load"] - b["load"]) <= 13.0


def test_a_rank_that_leaves_is_noticed_by_the_other():
    outs = _run("leave")
    by_rank = {o[1]["rank"]: o for o in outs if o[1] is not None}
    assert 0 in by_rank, outs
    code, res, _ = by_rank[0]
    assert code != 0 and res.get("error"), outs


def test_single_process_needs_no_group():
    assert MG.rank_info({}) == (0, 0, 1)
    assert MG.init("gloo", 1) is None
    assert MG.max_over_ranks(3.5, None) == 3.5
    assert MG.job_throughput(100, 4, 2.0) == 200000.0


def test_shard_is_a_balanced_partition():
    costs = [float(c) for c in (9, 1, 1, 1, 8, 2, 2, 7, 3, 3)]
    parts = [MG.shard(costs, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
