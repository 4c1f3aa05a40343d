"""x-slab decomposition of a hydrodynamics-only run.

The reference splits its grid along x over MPI ranks (Grid::initialise,
src/Fluid/Grid.cpp:446-459), fills the ghost cells of a face between two
ranks from the neighbour (Grid::applyBCs, PARTITION, Grid.cpp:804-833) and
takes the minimum time step over ranks (Torch::calculateTimeStep,
src/Torch/Torch.cpp:323-335).  Here every slab is a library context made by
trg_create_slab; the library packs the slab's boundary layers before each
flux computation and calls a host hook, which moves them between slabs and
takes the time-step minimum over slabs:

* ``DistributedSlab``: one slab per process and GPU, the hook on
  ``torch.distributed`` (NCCL over NVLink between GPUs; point-to-point
  send/recv of the halos, an all-reduce MIN of the time-step minima), all
  enqueued on the library's stream.
* ``LocalSlabs``: every slab of a run in one process on one GPU, each stepped
  by its own host thread; the hook copies the halos between the slabs'
  buffers on the device, ordered by CUDA events (no kernel waits on another).

The exchange pattern itself (``exchange_halos``, ``min_over_slabs``) is plain
``torch.distributed`` and runs on CPU tensors too (gloo), where the tests
check it.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import EXCHANGE_DT, EXCHANGE_FN, EXCHANGE_HALO, PRECISION_FP32, PRECISION_FP64, Torch, TrgError, \
    _ptr, load_library, make_params


def slab_ranges(nx: int, nslabs: int) -> List[Tuple[int, int]]:
    """(x0, width) of each slab: nx // nslabs cells each, the last nx % nslabs
    slabs one more (calcCoreCells / calcLeftBoundaryPosition, Grid.cpp:446-459)."""
    if nslabs < 1 or nx < 2 * nslabs:
        raise ValueError("every slab needs at least two x layers")
    base, extra = divmod(nx, nslabs)
    out, x0 = [], 0
    for r in range(nslabs):
        w = base + (1 if nslabs - r <= extra else 0)
        out.append((x0, w))
        x0 += w
    return out


def neighbours(rank: int, nslabs: int, periodic: bool) -> Tuple[Optional[int], Optional[int]]:
    """Ranks of the low-x and high-x neighbours (None at a grid end unless periodic)."""
    left = rank - 1 if rank > 0 else (nslabs - 1 if periodic and nslabs > 1 else None)
    right = rank + 1 if rank < nslabs - 1 else (0 if periodic and nslabs > 1 else None)
    return left, right


def f32_scales(tp, ic) -> np.ndarray:
    """The whole grid's reference density and pressure of the FP32 form (code
    units), which every slab of a run takes so that all scale their state
    alike (host only)."""
    lib = load_library()
    p = make_params(tp, ic.side_length, ic.ncells, PRECISION_FP32, 0)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
            (ic.den, ic.pre, ic.hii, ic.vel[0], ic.vel[1], ic.vel[2])]
    out = np.zeros(2)
    rc = lib.trg_f32_scales(C.byref(p), *[_ptr(a) for a in arrs], _ptr(out))
    if rc:
        raise TrgError(rc, "trg_f32_scales: the grid is refused")
    return out


def exchange_halos(send, recv, left, right, group=None):
    """One halo exchange of a slab: recv[0] (low-x ghosts) from the left
    neighbour's send[1], recv[1] from the right neighbour's send[0], as
    point-to-point send/recv (None: no neighbour on that side).  send and
    recv are [2, ...] tensors (side first)."""
    import torch.distributed as dist
    ops = []
    if left is not None:
        ops += [dist.P2POp(dist.isend, send[0], left, group), dist.P2POp(dist.irecv, recv[0], left, group)]
    if right is not None:
        ops += [dist.P2POp(dist.isend, send[1], right, group), dist.P2POp(dist.irecv, recv[1], right, group)]
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()


def min_over_slabs(t, group=None):
    """The time-step minima (int64 bit patterns of positive doubles) become
    their minimum over all slabs."""
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)


class _SlabBuffers:
    """A slab's device buffers: halo send and receive [2 sides, 2 layers, 7
    fields, ny*nz] and the three time-step minima."""

    def __init__(self, sim: Torch, device):
        import torch
        nbytes = int(sim.lib.trg_slab_halo_bytes(sim.ctx))
        dtype = torch.float32 if sim.fp32_state else torch.float64
        n = nbytes // (4 if sim.fp32_state else 8)
        self.send = torch.zeros((2, n // 2), dtype=dtype, device=device)
        self.recv = torch.zeros((2, n // 2), dtype=dtype, device=device)
        self.dt = torch.zeros(3, dtype=torch.int64, device=device)
        self.parts = int(sim.lib.trg_slab_partitions(sim.ctx))


def _is_fp32_state(tp, precision) -> bool:
    return precision == PRECISION_FP32 and not (tp.radiation_on or tp.cooling_on)


class DistributedSlab:
    """This process's slab of a decomposed run: rank `rank` of `world`, on
    CUDA device `device`, exchanging over the default process group (NCCL)."""

    def __init__(self, tp, ic, rank: int, world: int, precision: int = PRECISION_FP64, device: int = 0,
                 scales=None):
        import torch
        self.rank, self.world = rank, world
        self.ranges = slab_ranges(int(ic.ncells[0]), world)
        x0, nx = self.ranges[rank]
        if precision == PRECISION_FP32 and scales is None:
            scales = f32_scales(tp, ic)
        self.sim = Torch(tp, ic, precision=precision, device=device, slab=(x0, nx, scales))
        self.sim.fp32_state = _is_fp32_state(tp, precision)
        self.buf = _SlabBuffers(self.sim, torch.device("cuda", device))
        left, right = neighbours(rank, world, True)
        self.left = left if self.buf.parts & 1 else None
        self.right = right if self.buf.parts & 2 else None
        self.device = device
        self._fn = EXCHANGE_FN(self._hook)
        rc = self.sim.lib.trg_slab_exchange(self.sim.ctx, self._fn, None, C.c_void_p(self.buf.send.data_ptr()),
                                            C.c_void_p(self.buf.recv.data_ptr()), C.c_void_p(self.buf.dt.data_ptr()))
        if rc:
            raise TrgError(rc, self.sim.lib.trg_last_error(self.sim.ctx).decode())

    def _hook(self, user, what, stream):
        import torch
        try:
            s = torch.cuda.ExternalStream(stream, device=torch.device("cuda", self.device))
            with torch.cuda.stream(s):
                if what == EXCHANGE_HALO:
                    exchange_halos(self.buf.send, self.buf.recv, self.left, self.right)
                elif what == EXCHANGE_DT:
                    min_over_slabs(self.buf.dt)
            return 0
        except Exception:
            return 1

    def run_steps(self, nsteps: int, dt_next: Optional[float] = None):
        return self.sim.run_steps(nsteps, dt_next)

    def close(self):
        self.sim.close()


class LocalSlabs:
    """Every slab of a decomposed run in this process, on one CUDA device:
    slab r steps in host thread r; its hook meets the others at a barrier and
    copies the neighbours' halos into its receive buffer on its own stream
    after their packs (CUDA events), and no slab packs again before its
    neighbours have copied (events again).  The time-step minima are reduced
    the same way.  No kernel waits on another."""

    def __init__(self, tp, ic, nslabs: int, precision: int = PRECISION_FP64, device: int = 0, timeout: float = 120.0):
        import torch
        self.n = nslabs
        self.ranges = slab_ranges(int(ic.ncells[0]), nslabs)
        self.ny, self.nz = int(ic.ncells[1]), int(ic.ncells[2])
        scales = f32_scales(tp, ic) if precision == PRECISION_FP32 else None
        self.dev = torch.device("cuda", device)
        self.sims, self.bufs = [], []
        for x0, nx in self.ranges:
            sim = Torch(tp, ic, precision=precision, device=device, slab=(x0, nx, scales))
            sim.fp32_state = _is_fp32_state(tp, precision)
            self.sims.append(sim)
            self.bufs.append(_SlabBuffers(sim, self.dev))
        self.barrier = threading.Barrier(nslabs, timeout=timeout)
        self.ev_pack = [torch.cuda.Event() for _ in range(nslabs)]
        self.ev_copy = [torch.cuda.Event() for _ in range(nslabs)]
        self.nb = []
        for r in range(nslabs):
            left, right = neighbours(r, nslabs, True)
            parts = self.bufs[r].parts
            self.nb.append((left if parts & 1 else None, right if parts & 2 else None))
        self._fns = []
        for r, sim in enumerate(self.sims):
            fn = EXCHANGE_FN(lambda user, what, stream, r=r: self._hook(r, what, stream))
            self._fns.append(fn)
            b = self.bufs[r]
            rc = sim.lib.trg_slab_exchange(sim.ctx, fn, None, C.c_void_p(b.send.data_ptr()),
                                           C.c_void_p(b.recv.data_ptr()), C.c_void_p(b.dt.data_ptr()))
            if rc:
                raise TrgError(rc, sim.lib.trg_last_error(sim.ctx).decode())

    def _hook(self, r: int, what: int, stream) -> int:
        import torch
        try:
            s = torch.cuda.ExternalStream(stream, device=self.dev)
            left, right = self.nb[r]
            others = [q for q in (left, right) if q is not None]
            if what == EXCHANGE_DT:
                others = [q for q in range(self.n) if q != r]
            self.ev_pack[r].record(s)
            self.barrier.wait()
            with torch.cuda.stream(s):
                for q in others:
                    s.wait_event(self.ev_pack[q])
                if what == EXCHANGE_HALO:
                    if left is not None:
                        self.bufs[r].recv[0].copy_(self.bufs[left].send[1], non_blocking=True)
                    if right is not None:
                        self.bufs[r].recv[1].copy_(self.bufs[right].send[0], non_blocking=True)
                else:
                    m = torch.stack([self.bufs[q].dt for q in range(self.n)]).min(dim=0).values
                    self._dt_min = getattr(self, "_dt_min", {})
                    self._dt_min[r] = m
                self.ev_copy[r].record(s)
            self.barrier.wait()
            with torch.cuda.stream(s):
                for q in others:
                    s.wait_event(self.ev_copy[q])
                if what == EXCHANGE_DT:
                    self.bufs[r].dt.copy_(self._dt_min[r], non_blocking=True)
            return 0
        except Exception:
            self.barrier.abort()
            return 1

    def run_steps(self, nsteps: int, dt_next: Optional[float] = None):
        """nsteps full steps of every slab, each slab in its own thread."""
        errors = [None] * self.n

        def work(r):
            try:
                self.sims[r].run_steps(nsteps, dt_next)
            except Exception as e:  # reported after every thread has ended
                errors[r] = e
                self.barrier.abort()

        threads = [threading.Thread(target=work, args=(r,)) for r in range(self.n)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for e in errors:
            if e is not None:
                raise e

    def state(self):
        """The whole grid's conserved and primitive states ([7][N] each),
        assembled from the slabs, and the slabs' times."""
        sts = [sim.state() for sim in self.sims]
        widths = [nx for _, nx in self.ranges]
        return (assemble([st.U for st in sts], widths, self.ny, self.nz),
                assemble([st.Q for st in sts], widths, self.ny, self.nz), [st.time for st in sts])

    def close(self):
        for sim in self.sims:
            sim.close()


def assemble(fields: Sequence[np.ndarray], widths: Sequence[int], ny: int, nz: int) -> np.ndarray:
    """Fields [k][N_slab] of the slabs side by side along x -> [k][N]."""
    blocks = [f.reshape(f.shape[0], nz, ny, w) for f, w in zip(fields, widths)]
    out = np.concatenate(blocks, axis=3)
    return out.reshape(out.shape[0], -1)
