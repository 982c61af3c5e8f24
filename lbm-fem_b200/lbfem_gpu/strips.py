"""y-strip decomposition of one mesh over several contexts (one per rank).

The reference distributes its triangulation and vectors over MPI ranks
(discretization.h:71-75), exchanges ghost values inside every operator
application (MatrixFree::loop, advection.h:151-175) and sums every CG dot
product over the ranks (mass.h:204-211). Here the mesh is cut into strips of
whole cell rows. Rank r owns the node rows of its cells and keeps, below them,
one ghost cell layer (`degree` node rows) and, above them, the neighbour's
first node row: exactly what an owned node's operator rows touch. Each rank's
context is built on that local mesh (non-periodic in y) and told its ghost
rows with lbfem_gpu_set_strip; the library then exchanges the ghost rows of
the CG residual (or of the lumped / iterated-lumping increment) and sums the
solver's dot products through the callback installed here. Nodal maps and the
streaming right-hand side need no exchange: a ghost row's populations are
updated by the same pointwise arithmetic as on their owner, from exchanged
increments.

Communicators: ``DistComm`` (torch.distributed point-to-point and all_reduce;
gloo with host buffers, NCCL with device buffers) and ``LocalComm`` (all ranks
in one process, one host thread each, copies between the ranks' buffers; no
kernel of one rank waits on another's).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading

import numpy as np

from . import cases

COMM_EXCHANGE, COMM_ALLREDUCE = 0, 1
COMM_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int64)


class StripDesc(C.Structure):
    _fields_ = [("ghost_below", C.c_int32), ("ghost_above", C.c_int32), ("cell_below", C.c_double),
                ("cell_above", C.c_double), ("comm", COMM_FN), ("user", C.c_void_p),
                ("send_below", C.c_void_p), ("send_above", C.c_void_p), ("recv_below", C.c_void_p),
                ("recv_above", C.c_void_p), ("sums", C.POINTER(C.c_double))]


@dataclasses.dataclass
class Strip:
    """Rank `rank`'s part of a mesh: its cell rows [cy0, cy1), the local mesh
    (its cells, plus the ghost cell layer below when it has a neighbour there,
    non-periodic in y, with the walls of its rows) and the map of local node
    rows to global ones."""

    rank: int
    n_ranks: int
    cy0: int
    cy1: int
    below: int | None  # neighbour ranks (None: a wall)
    above: int | None
    ghost_below: int
    ghost_above: int
    cell_below: float
    cell_above: float
    mesh: cases.Mesh
    rows: np.ndarray  # global node row of every local node row

    @property
    def own_rows(self):
        """Local node rows this rank owns."""
        return slice(self.ghost_below, self.mesh.nfy - self.ghost_above)

    def local_index(self, mesh):
        """Global structured index of every local node (local structured order)."""
        return (self.rows[:, None] * mesh.nfx + np.arange(mesh.nfx)[None, :]).ravel()

    def owned_index(self, mesh):
        """(local, global) structured indices of the owned nodes."""
        nfx = mesh.nfx
        lr = np.arange(self.mesh.nfy)[self.own_rows]
        loc = (lr[:, None] * nfx + np.arange(nfx)[None, :]).ravel()
        glo = (self.rows[lr][:, None] * nfx + np.arange(nfx)[None, :]).ravel()
        return loc, glo


def partition(mesh: cases.Mesh, n_ranks: int) -> list[Strip]:
    """Strips of whole cell rows, as even as the cell count allows; every strip
    needs at least 2 cell rows."""
    P, ncy = mesh.degree, mesh.n_cells_y
    if n_ranks < 2 or ncy < 2 * n_ranks:
        raise ValueError(f"{n_ranks} strips of {ncy} cell rows: at least 2 ranks and 2 cell rows each")
    vy = np.asarray(mesh.vertex_y, float)
    L = vy[-1] - vy[0]
    hy = np.diff(vy)
    periodic = bool(mesh.periodic_y)
    nuy = P * ncy  # distinct node rows of a periodic axis
    wall_rows = {}
    for k, dof in enumerate(np.asarray(mesh.wall_dof, np.int64)):
        wall_rows.setdefault(int(dof) // mesh.nfx, []).append((int(dof) % mesh.nfx, mesh.wall_velocity[k]))
    out = []
    for r in range(n_ranks):
        cy0, cy1 = r * ncy // n_ranks, (r + 1) * ncy // n_ranks
        below = (r - 1) % n_ranks if (periodic or r > 0) else None
        above = (r + 1) % n_ranks if (periodic or r < n_ranks - 1) else None
        lc0 = cy0 - (1 if below is not None else 0)
        cells = np.arange(lc0, cy1 + 1)  # vertex indices of the local cells, possibly -1 (periodic wrap)
        lvy = vy[cells % ncy] + L * np.floor_divide(cells, ncy)
        lvy[cells == ncy] = vy[ncy]
        nrow = P * (cy1 - lc0) + 1
        rows = P * lc0 + np.arange(nrow)
        if periodic:
            rows = rows % nuy
        lm = cases.Mesh(P, mesh.n_cells_x, cy1 - lc0, mesh.periodic_x, False, np.asarray(mesh.vertex_x, float),
                        lvy, mesh.h_min)
        wd, wv = [], []
        for lr, gr in enumerate(rows):
            for i, vel in wall_rows.get(int(gr), []):
                wd.append(lr * mesh.nfx + i)
                wv.append(vel)
        lm.wall_dof = np.asarray(wd, np.int64)
        lm.wall_velocity = np.asarray(wv, float).reshape(-1, 2)
        out.append(Strip(r, n_ranks, cy0, cy1, below, above, P if below is not None else 0,
                         1 if above is not None else 0,
                         float(hy[(lc0 - 1) % ncy]) if below is not None else 0.0,
                         float(hy[cy1 % ncy]) if above is not None else 0.0, lm, rows))
    return out


class _Buffers:
    """The exchange buffers and the sums buffer of one rank (torch tensors: on
    the rank's GPU for the CUDA library, in host memory for the oracle)."""

    def __init__(self, nbytes, device):
        import torch

        mk = lambda: torch.zeros(nbytes, dtype=torch.uint8, device=device)  # noqa: E731
        self.send_below, self.send_above, self.recv_below, self.recv_above = mk(), mk(), mk(), mk()
        self.sums = torch.zeros(64, dtype=torch.float64, device=device)


class DistComm:
    """The collectives of one rank over a torch.distributed process group."""

    def __init__(self, strip: Strip, bufs: _Buffers, group=None):
        self.strip, self.bufs, self.group = strip, bufs, group

    def __call__(self, op, count):
        import torch
        import torch.distributed as dist

        b, s = self.bufs, self.strip
        P = s.mesh.degree
        if op == COMM_ALLREDUCE:
            dist.all_reduce(b.sums[:count], group=self.group)
        else:
            # sends first, then receives, in this order on every rank: with two
            # ranks on a periodic axis both neighbours are the same rank, and its
            # two messages are told apart by order (and tag)
            ops = []
            if s.below is not None:
                ops.append(dist.P2POp(dist.isend, b.send_below[:count], s.below, self.group, tag=0))
            if s.above is not None:
                ops.append(dist.P2POp(dist.isend, b.send_above[:P * count], s.above, self.group, tag=1))
            if s.above is not None:
                ops.append(dist.P2POp(dist.irecv, b.recv_above[:count], s.above, self.group, tag=0))
            if s.below is not None:
                ops.append(dist.P2POp(dist.irecv, b.recv_below[:P * count], s.below, self.group, tag=1))
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if b.sums.is_cuda:
            torch.cuda.current_stream(b.sums.device).synchronize()
        return 0


class LocalComm:
    """The collectives of n ranks that live in one process, one host thread each:
    a barrier, copies out of the neighbours' send buffers, a barrier. Sums are
    added in rank order (the same result on every rank)."""

    def __init__(self, strips: list[Strip], bufs: list[_Buffers]):
        self.strips, self.bufs = strips, bufs
        self.barrier = threading.Barrier(len(strips))

    def for_rank(self, r):
        return lambda op, count: self._call(r, op, count)

    def _call(self, r, op, count):
        import torch

        s, b = self.strips[r], self.bufs[r]
        P = s.mesh.degree
        self.barrier.wait()  # every rank's send buffers / sums are in place
        if op == COMM_ALLREDUCE:
            total = self.bufs[0].sums[:count].clone()
            for q in range(1, len(self.bufs)):
                total += self.bufs[q].sums[:count]
        else:
            if s.below is not None:
                b.recv_below[:P * count].copy_(self.bufs[s.below].send_above[:P * count])
            if s.above is not None:
                b.recv_above[:count].copy_(self.bufs[s.above].send_below[:count])
        if b.sums.is_cuda:
            torch.cuda.current_stream(b.sums.device).synchronize()
        self.barrier.wait()  # every rank has read the others' buffers
        if op == COMM_ALLREDUCE:
            b.sums[:count].copy_(total)
            if b.sums.is_cuda:
                torch.cuda.current_stream(b.sums.device).synchronize()
        return 0


class StripSolver:
    """Rank `strip.rank`'s context on its local mesh, with the collectives of
    `comm` (a callable (op, count) -> int). `make(mesh, params)` creates the
    context (lbfem_gpu.Solver, or the oracle's handle); `device`: where the
    exchange buffers live ("cuda:k" for the CUDA library, "cpu" for the oracle)."""

    def __init__(self, mesh: cases.Mesh, strip: Strip, params, make, device, comm_factory):
        self.global_mesh, self.strip = mesh, strip
        self.h = make(strip.mesh, params)
        nbytes = C.c_int64()
        self.h._call("strip_buffer_bytes", self.h.h, C.byref(nbytes))
        self.bufs = _Buffers(int(nbytes.value), device)
        self.comm = comm_factory(self)
        self._cb = COMM_FN(lambda user, op, count: self._dispatch(op, count))
        b = self.bufs
        desc = StripDesc(strip.ghost_below, strip.ghost_above, strip.cell_below, strip.cell_above, self._cb, None,
                         b.send_below.data_ptr(), b.send_above.data_ptr(), b.recv_below.data_ptr(),
                         b.recv_above.data_ptr(), C.cast(b.sums.data_ptr(), C.POINTER(C.c_double)))
        self.h._call("set_strip", self.h.h, C.byref(desc))

    def _dispatch(self, op, count):
        try:
            return int(self.comm(op, count))
        except Exception:  # an exception must not cross the C callback
            return 1

    # -- the Scheme interface on the global numbering
    def set_time_step(self, dt, lam):
        self.h.set_time_step(dt, lam)

    def _local(self, f_global):
        return np.ascontiguousarray(np.asarray(f_global)[:, self.strip.local_index(self.global_mesh)])

    def set_initial_populations(self, f_global):
        self.h.set_initial_populations(self._local(f_global))

    def set_populations(self, f_global):
        self.h.set_populations(self._local(f_global))

    def step(self, n=1):
        self.h.step(n)

    def owned_populations(self):
        """(global structured indices, populations there) of the owned nodes."""
        loc, glo = self.strip.owned_index(self.global_mesh)
        return glo, self.h.get_populations()[:, loc]

    def conservation_local(self):
        """This rank's share of the conservation sums (owned rows only)."""
        return self.h.conservation()

    def close(self):
        self.h.close()


def assemble(mesh: cases.Mesh, parts):
    """The global population array from every rank's owned_populations(); a
    periodic image row (owned by no rank) takes its source row's values, as
    after deal.II's constraints.distribute."""
    f = np.full((9, mesh.n_dofs), np.nan)
    for glo, vals in parts:
        f[:, glo] = vals
    if mesh.periodic_y:
        f[:, (mesh.nfy - 1) * mesh.nfx:] = f[:, :mesh.nfx]
    return f


def local_ranks(mesh, params, n_ranks, make, device):
    """n_ranks StripSolvers in this process with a LocalComm: the strips of one
    mesh on one device (each rank's step runs on its own host thread)."""
    strips = partition(mesh, n_ranks)
    holder = {}

    def factory(r):
        def comm_factory(solver):
            holder.setdefault("bufs", [None] * n_ranks)[r] = solver.bufs
            return lambda op, count: holder["comm"].for_rank(r)(op, count)
        return comm_factory

    solvers = [StripSolver(mesh, strips[r], params, make, device, factory(r)) for r in range(n_ranks)]
    holder["comm"] = LocalComm(strips, holder["bufs"])
    return solvers


def run_local(solvers, fn):
    """Calls fn(solver) for every rank on its own thread (collective calls such
    as step); re-raises the first exception."""
    errs = [None] * len(solvers)

    def body(k):
        try:
            fn(solvers[k])
        except BaseException as e:  # noqa: BLE001
            errs[k] = e

    ts = [threading.Thread(target=body, args=(k,)) for k in range(len(solvers))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for e in errs:
        if e is not None:
            raise e
