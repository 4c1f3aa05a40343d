"""x-slab decomposition of a run.

The reference splits its grid along x over MPI ranks (Grid::initialise,
src/Fluid/Grid.cpp:446-459), fills the ghost cells of a face between two
ranks from the neighbour (Grid::applyBCs, PARTITION, Grid.cpp:804-833),
takes the minimum time step over ranks (Torch::calculateTimeStep,
src/Torch/Torch.cpp:323-335) and, with a star, runs its causal sweeps rank
after rank outwards from the star's rank, each passing its boundary layer of
optical depths or column densities on (Radiation::transferRadiation,
src/Integrators/Radiation.cpp:573-636; Thermodynamics::rayTrace,
Thermodynamics.cpp:365-417).  Here every slab is a library context made by
trg_create_slab; the library packs the slab's boundary layers before each
flux computation and after each causal sweep and calls a host hook, which
moves them between slabs and takes the time-step minimum over slabs:

* ``DistributedSlab``: one slab per process and GPU, the hook on
  ``torch.distributed`` (NCCL over NVLink between GPUs; point-to-point
  send/recv of the halos, an all-reduce MIN of the time-step minima), all
  enqueued on the library's stream.
* ``LocalSlabs``: every slab of a run in one process on one GPU, each stepped
  by its own host thread; the hook copies the halos between the slabs'
  buffers on the device, ordered by CUDA events (no kernel waits on another).

The exchange pattern itself (``exchange_halos``, ``min_over_slabs``,
``sweep_receive``, ``sweep_send``) is plain ``torch.distributed`` and runs on
CPU tensors too (gloo), where the tests check it.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import EXCHANGE_DT, EXCHANGE_FN, EXCHANGE_HALO, EXCHANGE_SWEEP_IN, EXCHANGE_SWEEP_OUT, PRECISION_FP32, \
    PRECISION_FP64, Torch, TrgError, _ptr, load_library, make_params


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


def sweep_upstream(rank: int, nslabs: int, star_side: int) -> Optional[int]:
    """The slab whose boundary layer a slab's causal sweep reads
    (trg_slab_star_side: 0 the star is in this slab, 1 at lower x, 2 at
    higher x): the neighbour on the star's side, None for the star's slab."""
    if star_side == 1:
        return rank - 1
    if star_side == 2:
        return rank + 1
    return None


def sweep_downstream(rank: int, nslabs: int, star_side: int) -> List[Tuple[int, int]]:
    """(neighbour, side of this slab's send buffer) of the slabs a slab hands
    its boundary layers to after a sweep: the low-x neighbour unless the star
    lies at lower x or this is the first slab, the high-x one unless it lies
    at higher x or this is the last (Radiation.cpp:614-635)."""
    out = []
    if star_side != 1 and rank > 0:
        out.append((rank - 1, 0))
    if star_side != 2 and rank < nslabs - 1:
        out.append((rank + 1, 1))
    return out


def sweep_receive(recv, rank, nslabs, star_side, group=None):
    """Before a sweep: recv[side facing the star] from the star-side
    neighbour's send buffer (point-to-point recv; nothing for the star's
    slab).  recv and send are [2, ...] tensors (side first)."""
    import torch.distributed as dist
    up = sweep_upstream(rank, nslabs, star_side)
    if up is not None:
        dist.recv(recv[0 if up < rank else 1], up, group)


def sweep_send(send, rank, nslabs, star_side, group=None):
    """After a sweep: this slab's boundary layers to the slabs away from the star."""
    import torch.distributed as dist
    for nb, side in sweep_downstream(rank, nslabs, star_side):
        dist.send(send[side], nb, group)


def min_over_slabs(t, group=None):
    """The time-step minima (int64 bit patterns of positive doubles) become
    their minimum over all slabs."""
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)


class _SlabBuffers:
    """A slab's device buffers: halo send and receive [2 sides, 2 layers, 7
    fields, ny*nz], the three time-step minima and, in a run with a star, the
    sweep send and receive buffers [2 sides, ny*nz*4] (registered here)."""

    def __init__(self, sim: Torch, device, star: bool):
        import torch
        nbytes = int(sim.lib.trg_slab_halo_bytes(sim.ctx))
        dtype = torch.float32 if sim.fp32_state else torch.float64
        n = nbytes // (4 if sim.fp32_state else 8)
        self.send = torch.zeros((2, n // 2), dtype=dtype, device=device)
        self.recv = torch.zeros((2, n // 2), dtype=dtype, device=device)
        self.dt = torch.zeros(3, dtype=torch.int64, device=device)
        self.parts = int(sim.lib.trg_slab_partitions(sim.ctx))
        self.star_side = int(sim.lib.trg_slab_star_side(sim.ctx))
        self.sweeps = bool(star and self.parts)
        if self.sweeps:
            m = int(sim.lib.trg_slab_sweep_bytes(sim.ctx)) // 8
            self.sw_send = torch.zeros((2, m // 2), dtype=torch.float64, device=device)
            self.sw_recv = torch.zeros((2, m // 2), dtype=torch.float64, device=device)
            rc = sim.lib.trg_slab_sweep_exchange(sim.ctx, C.c_void_p(self.sw_send.data_ptr()),
                                                 C.c_void_p(self.sw_recv.data_ptr()))
            if rc:
                raise TrgError(rc, sim.lib.trg_last_error(sim.ctx).decode())


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
        self.buf = _SlabBuffers(self.sim, torch.device("cuda", device), tp.star_on)
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
                elif what == EXCHANGE_SWEEP_IN:
                    sweep_receive(self.buf.sw_recv, self.rank, self.world, self.buf.star_side)
                elif what == EXCHANGE_SWEEP_OUT:
                    sweep_send(self.buf.sw_send, self.rank, self.world, self.buf.star_side)
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
    the same way.  With a star, a slab's hook before a causal sweep waits (on
    the host, with a time limit) until the star-side neighbour has packed
    that sweep's boundary layer and copies it after the pack (an event), and
    until the neighbours away from the star have copied its previous one,
    whose copies its next pack then follows (events): the slabs sweep one
    after another outwards from the star, as the reference's ranks do.  No
    kernel waits on another."""

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
            self.bufs.append(_SlabBuffers(sim, self.dev, tp.star_on))
        self.timeout = timeout
        self.barrier = threading.Barrier(nslabs, timeout=timeout)
        # causal sweeps: per slab the sweeps begun, the boundary layers packed
        # and the star-side layers copied (host counters under one condition),
        # with the events of the latest pack and copy
        self.sw_cond = threading.Condition()
        self.sw_broken = False
        self.sw_begun = [0] * nslabs
        self.sw_packed = [0] * nslabs
        self.sw_copied = [0] * nslabs
        self.ev_sw_pack = [torch.cuda.Event() for _ in range(nslabs)]
        self.ev_sw_copy = [torch.cuda.Event() for _ in range(nslabs)]
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

    def _sw_wait(self, pred):
        """Waits (host) under the sweep condition until pred() holds."""
        if not self.sw_cond.wait_for(lambda: self.sw_broken or pred(), timeout=self.timeout) or self.sw_broken:
            raise RuntimeError("slab sweep exchange: a neighbour did not arrive in time")

    def _sweep_hook(self, r: int, what: int, s) -> None:
        import torch
        b = self.bufs[r]
        if what == EXCHANGE_SWEEP_OUT:
            self.ev_sw_pack[r].record(s)
            with self.sw_cond:
                self.sw_packed[r] += 1
                self.sw_cond.notify_all()
            return
        k = self.sw_begun[r]  # this sweep's index
        with self.sw_cond:
            # the neighbours away from the star have copied this slab's last layers
            for d, _ in sweep_downstream(r, self.n, b.star_side):
                self._sw_wait(lambda d=d: self.sw_copied[d] >= k)
                if k > 0:
                    s.wait_event(self.ev_sw_copy[d])
            up = sweep_upstream(r, self.n, b.star_side)
            if up is not None:
                self._sw_wait(lambda: self.sw_packed[up] >= k + 1)
                s.wait_event(self.ev_sw_pack[up])
        if up is not None:
            side = 0 if up < r else 1
            with torch.cuda.stream(s):
                b.sw_recv[side].copy_(self.bufs[up].sw_send[1 - side], non_blocking=True)
            self.ev_sw_copy[r].record(s)
            with self.sw_cond:
                self.sw_copied[r] = k + 1
                self.sw_cond.notify_all()
        self.sw_begun[r] = k + 1

    def _hook(self, r: int, what: int, stream) -> int:
        import torch
        try:
            s = torch.cuda.ExternalStream(stream, device=self.dev)
            if what in (EXCHANGE_SWEEP_IN, EXCHANGE_SWEEP_OUT):
                self._sweep_hook(r, what, s)
                return 0
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
            with self.sw_cond:
                self.sw_broken = True
                self.sw_cond.notify_all()
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
                with self.sw_cond:
                    self.sw_broken = True
                    self.sw_cond.notify_all()

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

    def full_state(self):
        """The whole grid's U, Q, R and T ([k][N] each, R and T field after
        field), assembled from the slabs, and each slab's state (time, time
        steps)."""
        sts = [sim.state() for sim in self.sims]
        widths = [nx for _, nx in self.ranges]

        def whole(name):
            return assemble([getattr(st, name) for st in sts], widths, self.ny, self.nz)
        return whole("U"), whole("Q"), whole("R"), whole("T"), sts

    def close(self):
        for sim in self.sims:
            sim.close()


def assemble(fields: Sequence[np.ndarray], widths: Sequence[int], ny: int, nz: int) -> np.ndarray:
    """Fields [k][N_slab] of the slabs side by side along x -> [k][N]."""
    blocks = [f.reshape(f.shape[0], nz, ny, w) for f, w in zip(fields, widths)]
    out = np.concatenate(blocks, axis=3)
    return out.reshape(out.shape[0], -1)
