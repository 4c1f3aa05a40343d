"""The N > 1 path of bench.py on CPU: gloo ranks (world size 2) synchronise,
max-reduce their timings, and the reference arm runs on rank 0 only."""
import os
import socket
import sys
import types

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup(backend="gloo")
    bench.barrier(pg)
    m = bench.max_over_ranks(pg, 10.0 * (r + 1), local)
    rc = 0
    if r != 0:  # the reference arm: ranks other than 0 exit without work
        rc = bench.run_reference_arm(types.SimpleNamespace(), r)
    bench.barrier(pg)
    pg.destroy_process_group()
    out.put((r, w, m, rc))


def test_two_gloo_ranks_reduce_and_reference_arm_on_rank0():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1]
    assert all(w == 2 and m == 20.0 and rc == 0 for _, w, m, rc in res)


def test_reference_arm_line_names_its_sample(capsys):
    """The reference arm's JSON line: the workload's metric, measured on a
    bounded sample that the line itself names (grid size and process count)."""
    import json
    sys.path.insert(0, ROOT)
    import bench
    args = types.SimpleNamespace(workload="hii", n=256, steps=1, warmup=0, gpus=1)
    assert bench.run_reference_arm(args, 0) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert "sample" in line["config"]["workload"] and "32^3" in line["config"]["workload"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] >= 1
