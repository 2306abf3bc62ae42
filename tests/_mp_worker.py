"""One rank of the multi-process tests (launched by test_multiprocess.py with
RANK / WORLD_SIZE / MASTER_* set, as torchrun would): joins a gloo group and
runs the cross-rank steps of a benchmark run, printing one JSON line."""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from map_b200 import multigpu as MG  # noqa: E402


def main():
    mode = sys.argv[1]
    rank, local, world = MG.rank_info()
    dist = MG.init("gloo", world, timeout_s=20)
    try:
        MG.barrier(dist)
        if mode == "leave" and rank == 1:
            os._exit(0)   # a rank that leaves between steps, with nothing in flight
        slowest = MG.max_over_ranks(10.0 + 5.0 * rank, dist)
        costs = [float((7 * i) % 13 + 1) for i in range(40)]
        mine = MG.shard(costs, rank, world)
        print(json.dumps({"rank": rank, "local": local, "world": world, "slowest_ms": slowest,
                          "gcells": MG.job_throughput(1e9, world, slowest) / 1e9, "shard": mine,
                          "load": sum(costs[i] for i in mine)}), flush=True)
        MG.finish(dist)
    except Exception as e:   # reported to the test, which checks the other rank noticed the failure
        print(json.dumps({"rank": rank, "error": type(e).__name__}), flush=True)
        sys.exit(3)


if __name__ == "__main__":
    main()
