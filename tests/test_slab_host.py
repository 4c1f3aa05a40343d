"""Host side of the x-slab decomposition on CPU: the slab widths follow the
reference's rule (Grid.cpp:446-459), and the exchange pattern the GPU hook
runs over torch.distributed - the halo send/recv between neighbours, with the
two ends joined for periodic grids, and the minimum of the time-step minima -
moves the right layers between three gloo ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_core_cells(nx, nproc, iproc):
    """calcCoreCells of the reference (Grid.cpp:446-452), restated."""
    ncells = nx // nproc
    cells_left = nx - nproc * ncells
    if nproc - iproc <= cells_left:
        ncells += 1
    return ncells


def test_slab_ranges_follow_the_reference_rule():
    sys.path.insert(0, ROOT)
    from torch_b200 import slabs
    for nx, n in ((10, 3), (256, 4), (257, 8), (150, 7), (4, 2)):
        r = slabs.slab_ranges(nx, n)
        assert [w for _, w in r] == [reference_core_cells(nx, n, i) for i in range(n)]
        assert r[0][0] == 0 and all(r[i][0] + r[i][1] == r[i + 1][0] for i in range(n - 1))
        assert r[-1][0] + r[-1][1] == nx
    with pytest.raises(ValueError):
        slabs.slab_ranges(5, 3)  # a slab needs two x layers (the ghost depth)
    assert slabs.neighbours(0, 3, False) == (None, 1) and slabs.neighbours(2, 3, False) == (1, None)
    assert slabs.neighbours(0, 3, True) == (2, 1) and slabs.neighbours(0, 1, True) == (None, None)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, periodic, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from torch_b200 import slabs
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # send[side] holds this rank's layers next to that face, tagged rank*10 + side
    send = torch.stack([torch.full((2, 7, 5), float(rank * 10 + side)) for side in (0, 1)])
    recv = torch.full_like(send, -1.0)
    left, right = slabs.neighbours(rank, world, periodic)
    slabs.exchange_halos(send, recv, left, right)
    dt = torch.tensor([100 + rank, 50 - rank, 7 * (rank + 1)], dtype=torch.int64)
    slabs.min_over_slabs(dt)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, left, right, float(recv[0].mean()), float(recv[1].mean()), dt.tolist()))


@pytest.mark.parametrize("periodic", [False, True])
def test_halo_exchange_pattern_on_three_gloo_ranks(periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 3
    ps = [ctx.Process(target=_rank, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, left, right, low, high, dt in res:
        # low-x ghosts: the left neighbour's high-x layers; high-x ghosts: the right neighbour's low-x layers
        assert low == (left * 10 + 1 if left is not None else -1.0)
        assert high == (right * 10 + 0 if right is not None else -1.0)
        assert dt == [100, 48, 7]


def _sweep_rank(rank, world, port, star_slab, out):
    """One rank of a chain of causal sweeps: each 'sweep' adds one to the
    value received from the star-side neighbour (the star's slab starts from
    its own rank), as a slab's boundary layer depends on its upstream one."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from torch_b200 import slabs
    dist.init_process_group("gloo", rank=rank, world_size=world)
    star_side = 0 if rank == star_slab else (1 if star_slab < rank else 2)
    recv = torch.full((2, 3, 4), -1.0)
    send = torch.zeros_like(recv)
    seen = []
    for sweep in range(3):
        slabs.sweep_receive(recv, rank, world, star_side)
        up = slabs.sweep_upstream(rank, world, star_side)
        base = 100.0 * sweep if up is None else float(recv[0 if up < rank else 1].mean())
        seen.append(base)
        send.fill_(base + 1.0)
        slabs.sweep_send(send, rank, world, star_side)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, star_side, seen))


@pytest.mark.parametrize("star_slab", [0, 1, 3])
def test_sweep_chain_runs_outwards_from_the_star_on_four_gloo_ranks(star_slab):
    """The radiation and column-density sweeps of a decomposed run: a slab
    receives its star-side neighbour's boundary layer before its sweep and
    hands its own to the slabs away from the star after it
    (Radiation.cpp:573-636), so slab r's sweep k sees the star slab's sweep k
    passed on |r - star| times; no slab sends towards the star."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 4
    ps = [ctx.Process(target=_sweep_rank, args=(r, world, port, star_slab, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, star_side, seen in res:
        assert star_side == (0 if rank == star_slab else (1 if star_slab < rank else 2))
        assert seen == [100.0 * k + abs(rank - star_slab) for k in range(3)]


def test_sweep_neighbours():
    sys.path.insert(0, ROOT)
    from torch_b200 import slabs
    # star in slab 1 of 4: slab 1 sends both ways, 0 sends nowhere, 2 sends right, 3 nowhere
    assert slabs.sweep_downstream(1, 4, 0) == [(0, 0), (2, 1)]
    assert slabs.sweep_downstream(0, 4, 2) == [] and slabs.sweep_upstream(0, 4, 2) == 1
    assert slabs.sweep_downstream(2, 4, 1) == [(3, 1)] and slabs.sweep_upstream(2, 4, 1) == 1
    assert slabs.sweep_downstream(3, 4, 1) == [] and slabs.sweep_upstream(1, 4, 0) is None
