"""z-slab decomposition of the time step over processes, one GPU each.

The reference splits z over MPI ranks (Mpi_division.f90:6-24), exchanges
halo planes with MPI_SENDRECV before the predictor (two planes of u, v, w,
main.f90:163-183), after it (one plane of w*, main.f90:220-226), at every SOR
iteration (one plane of p, GS.f90:20-28) and after the solve (one plane of p,
main.f90:236-242), and takes the max of the sweep changes over the ranks
(MPI_ALLREDUCE, GS.f90:70).

Here each rank owns a slab context of the library (``include/ntcfd.h``,
``ntcfd_slab_stage``): the slab's nz, its slice of the z metrics and
coordinates, and ``NTCFD_BC_INTERFACE`` on each face it shares.  The driver
below runs the stages and moves the planes with ``torch.distributed``
point-to-point calls (NCCL between GPUs, gloo between CPU processes), so a
decomposed run repeats the single-domain FP64 red-black step bit for bit:

* red-black SOR needs the other colour's neighbours only, so one exchange of
  the just-updated colour after each half-sweep gives every slab the values
  a single domain would read (the reference exchanges once per lexicographic
  iteration instead, which changes its iterates with the rank count);
* the colour of a cell is that of its global (i+j+k): a slab whose first
  plane has an even global index runs the global red half-sweep with its own
  colour 1.

The slab's part of the work (``stage``, ``change``, ``get``, ``put``,
``sweep_field``) sits behind a small backend interface: ``LibrarySlab``
drives the CUDA library; tests drive the same exchange and stop logic with
a CPU restatement of the sweep on CPU ranks.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import abi
from .abi import (FIELD_E_BLACK, FIELD_E_RED, FIELD_P, FIELD_U, FIELD_V, FIELD_W, FIELD_WSTAR,
                  STAGE_CORRECT, STAGE_HALFSWEEP, STAGE_PREDICT, STAGE_PROJECT, STAGE_RHS, params_copy)


def partition(nz: int, nproc: int):
    """(gstart, gend, gcount) of every rank (Mpi_division.f90:6-24): the
    first nz mod nproc ranks take one plane more."""
    if nproc < 1 or nz < nproc:
        raise ValueError(f"cannot split {nz} planes over {nproc} ranks")
    zdv, zr = nz // nproc, nz - (nz // nproc) * nproc
    out = []
    for i in range(nproc):
        if i < zr:
            gs = 1 + i * (zdv + 1)
            ge = gs + zdv
        else:
            gs = 1 + i * zdv + zr
            ge = gs + zdv - 1
        out.append((gs, ge, ge - gs + 1))
    return out


def slab_grid(grid: dict, gs: int, ge: int) -> dict:
    """The slab's grid: x, y untouched; z metrics (entries k = -1..n+2) and
    node coordinates (k = -1..n+3) of global planes gs-2 .. ge+2 (+3)."""
    g = dict(grid)
    for name in ("iDz", "Dzs"):
        g[name] = np.ascontiguousarray(grid[name][gs - 1:ge + 4])
    g["Z"] = np.ascontiguousarray(grid["Z"][gs - 1:ge + 5])
    return g


def slab_halo(a: np.ndarray, gs: int, ge: int) -> np.ndarray:
    """Planes gs-2 .. ge+2 of a global halo array (nx+4, ny+4, nz+4)."""
    return np.asfortranarray(a[:, :, gs - 1:ge + 4])


def slab_params(params, rank: int, nproc: int, gcount: int):
    """The slab's parameters: its nz, and the interface kind on the faces
    it shares with a neighbour."""
    bc = [list(r) for r in params.bc]
    if nproc > 1 and abi.BC_PERIODIC in (bc[abi.BACK][0], bc[abi.FRONT][0]):
        raise ValueError("periodic z is not decomposed")
    if rank > 0:
        bc[abi.BACK] = [abi.BC_INTERFACE] * 3
    if rank < nproc - 1:
        bc[abi.FRONT] = [abi.BC_INTERFACE] * 3
    p = params_copy(params, nz=gcount)
    for w in range(6):
        for c in range(3):
            p.bc[w][c] = bc[w][c]
    return p


class SlabComm:
    """Neighbour exchanges and reductions of one rank (torch.distributed,
    initialised by the caller).  `device`: None for CPU tensors (gloo), or
    the CUDA device that NCCL moves the planes on."""

    def __init__(self, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.device = device

    def empty(self, n: int):
        t = self.torch
        return t.empty(n, dtype=t.float64, device=self.device if self.device is not None else "cpu")

    def exchange(self, backend, field: int, nplanes: int):
        """My first `nplanes` interior planes of `field` into the lower
        neighbour's top ghost planes, my last ones into the upper
        neighbour's bottom ghost planes; theirs into mine."""
        n, dist = backend.nz, self.dist
        lo, hi = self.rank - 1, self.rank + 1
        reqs, sends, recvs = [], [], []
        for nb, first, ghost in ((lo, 1, 1 - nplanes), (hi, n - nplanes + 1, n + 1)):
            if nb < 0 or nb >= self.size:
                continue
            out = backend.get(field, first, nplanes, self)
            buf = self.empty(nplanes * backend.plane_elems(field))
            sends.append(out)                   # alive until the sends complete
            reqs.append(dist.isend(out, nb))
            reqs.append(dist.irecv(buf, nb))
            recvs.append((ghost, buf))
        for r in reqs:
            r.wait()
        if self.device is not None:
            self.torch.cuda.synchronize(self.device)
        for k0, buf in recvs:
            backend.put(field, k0, buf)

    def max(self, x: float) -> float:
        t = self.torch.tensor([x], dtype=self.torch.float64,
                              device=self.device if self.device is not None else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


class LibrarySlab:
    """A slab context of the CUDA library (FP64)."""

    def __init__(self, params, grid: dict, rank: int, nproc: int):
        from .solver import Solver
        gs, ge, gc = partition(params.nz, nproc)[rank]
        if gc < 2:
            raise ValueError("each slab needs at least two planes (the two-plane velocity halo)")
        self.gs, self.ge, self.nz = gs, ge, gc
        self.solver = Solver(slab_params(params, rank, nproc, gc), slab_grid(grid, gs, ge))
        self.lib, self.h = self.solver.lib, self.solver.h

    def _check(self, rc):
        return self.solver._check(rc)

    def stage(self, stage: int, colour: int = 0):
        self._check(self.lib.ntcfd_slab_stage(self.h, stage, colour))

    def change(self) -> float:
        x = ctypes.c_double(0.0)
        self._check(self.lib.ntcfd_slab_change(self.h, ctypes.byref(x)))
        return x.value

    def plane_elems(self, field: int) -> int:
        return int(self.lib.ntcfd_slab_plane_elems(self.h, field))

    def get(self, field: int, k0: int, count: int, comm: SlabComm):
        buf = comm.empty(count * self.plane_elems(field))
        self._check(self.lib.ntcfd_slab_planes(self.h, field, k0, count, ctypes.c_void_p(buf.data_ptr()), 0))
        return buf

    def put(self, field: int, k0: int, buf):
        count = buf.numel() // self.plane_elems(field)
        self._check(self.lib.ntcfd_slab_planes(self.h, field, k0, count, ctypes.c_void_p(buf.data_ptr()), 1))

    @staticmethod
    def sweep_field(colour: int) -> int:
        return FIELD_E_BLACK if colour else FIELD_E_RED

    def close(self):
        self.solver.close()


class SlabRun:
    """One rank of a decomposed run: the exchanges and the stop rule of the
    time step around a slab backend."""

    def __init__(self, backend, comm: SlabComm, params):
        self.b, self.comm, self.prm = backend, comm, params
        self.flip = (backend.gs - 1) & 1       # local colour = global colour ^ flip

    def sor_solve(self):
        """GS.f90:9-79 over the slabs: sweeps, converged, last change."""
        b, c, P = self.b, self.comm, self.prm
        c.exchange(b, FIELD_P, 1)
        b.stage(STAGE_RHS)
        check = P.check_every if P.check_every > 0 else 1
        ik, ch, conv = 0, 0.0, False
        while ik < P.itmax:
            ik += 1
            for gcol in (0, 1):
                lc = gcol ^ self.flip
                b.stage(STAGE_HALFSWEEP, lc)
                c.exchange(b, b.sweep_field(lc), 1)
            ch = c.max(b.change())
            if math.isnan(ch):
                raise FloatingPointError("non-finite value in the SOR solve")
            if (ik % check == 0 or ik >= P.itmax) and not (ch > P.zeta):
                conv = True
                break
        b.stage(STAGE_CORRECT)
        c.exchange(b, FIELD_P, 1)
        return ik, conv, ch

    def step(self):
        """One time step (main.f90:139-259 without the force integral)."""
        b, c = self.b, self.comm
        for f in (FIELD_U, FIELD_V, FIELD_W):
            c.exchange(b, f, 2)
        b.stage(STAGE_PREDICT)
        c.exchange(b, FIELD_WSTAR, 1)
        out = self.sor_solve()
        b.stage(STAGE_PROJECT)
        return out
