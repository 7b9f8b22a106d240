"""The multi-rank bench path on the CPU: two gloo ranks (127.0.0.1), as
`torchrun --nproc-per-node 2 bench.py --gpus 2` starts them.  Each rank times
its own replica; the job's time is the maximum over ranks, which every rank
receives from one all-reduce (bench.max_over_ranks), and the reference arm
runs on rank 0 only."""
import os
import socket
import subprocess
import sys
import textwrap

from conftest import ROOT

SCRIPT = textwrap.dedent("""
    import os, sys, json, argparse
    sys.path.insert(0, {root!r})
    import torch.distributed as dist
    import bench

    def main():
        rank, world, _ = bench.dist_info()
        dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.5], world, "cpu")
        # the reference arm: rank 0 works, the others return at once
        args = argparse.Namespace(workload="none", steps=0, warmup=0)
        if rank != 0:
            bench.run_reference(args, rank, world)
        dist.barrier()
        dist.destroy_process_group()
        print(json.dumps({{"rank": rank, "max": got}}))

    if __name__ == "__main__":
        main()
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_with_two_gloo_ranks(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(SCRIPT.format(root=str(ROOT)))
    port = str(_free_port())
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(out.strip().splitlines()[-1])
    import json
    res = sorted((json.loads(o) for o in outs), key=lambda r: r["rank"])
    for r in res:
        assert r["max"] == [2.0, 10.0, 3.5]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1, "cpu") == [1.5, 2.5]
