"""z-slab decomposition (Mpi_division.f90:6-24, GS.f90:20-28,70) on CPU
ranks: the partition, the slab slices, and the decomposed red-black SOR solve
on three gloo ranks against the oracle's single-domain solve.

The ranks run the product's driver (``ntustcfdlab_b200.zslab.SlabRun``:
exchanges, colour flips, max over ranks, stop rule) around a CPU backend
defined here, which restates one half-sweep of GS.f90:35-68 over a slab in
numpy with the oracle's order of operations.  The CUDA backend of the same
driver is checked on the GPU in ``test_gpu_zslab.py``."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from ntustcfdlab_b200 import abi, zslab  # noqa: E402

N = (6, 5, 10)
SEED = 20261204


def test_partition_follows_mpi_division():
    assert zslab.partition(10, 3) == [(1, 4, 4), (5, 7, 3), (8, 10, 3)]
    assert zslab.partition(12, 4) == [(1, 3, 3), (4, 6, 3), (7, 9, 3), (10, 12, 3)]
    for nz in range(4, 40):
        for nproc in range(1, min(nz, 9) + 1):
            parts = zslab.partition(nz, nproc)
            assert parts[0][0] == 1 and parts[-1][1] == nz
            for (gs, ge, gc), (gs2, _, _) in zip(parts, parts[1:]):
                assert gs2 == ge + 1 and gc == ge - gs + 1
            sizes = [gc for _, _, gc in parts]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        zslab.partition(3, 4)


def test_slab_slices_and_params(orc):
    p = abi.make_params(*N, Re=100.0, dt=1e-3, bc={"Back": ("Dirichlet",) * 3})
    grid = orc.gridder_unequal(*N, 1.0, 2.0, 3.0, (12.5, 0.7, 1.3, 2, 2, 3, 3, 5, 0.4, 0.5, 0.9, 0.8, 1.6))
    for rank, (gs, ge, gc) in enumerate(zslab.partition(N[2], 3)):
        g = zslab.slab_grid(grid, gs, ge)
        for name in ("iDz", "Dzs"):
            assert len(g[name]) == gc + 4
            for k in range(-1, gc + 3):          # local k <-> global k + gs - 1
                assert g[name][k + 1] == grid[name][k + gs - 1 + 1]
        assert len(g["Z"]) == gc + 5 and g["Z"][2] == grid["Z"][gs + 1]
        sp = zslab.slab_params(p, rank, 3, gc)
        assert sp.nz == gc and sp.nx == N[0]
        assert (sp.bc[abi.BACK][0] == abi.BC_INTERFACE) == (rank > 0)
        assert (sp.bc[abi.FRONT][0] == abi.BC_INTERFACE) == (rank < 2)
        if rank == 0:
            assert list(sp.bc[abi.BACK]) == [abi.BC_DIRICHLET] * 3
    a = np.asfortranarray(np.arange(np.prod([n + 4 for n in N]), dtype=float).reshape([n + 4 for n in N], order="F"))
    s = zslab.slab_halo(a, 5, 7)
    assert s.shape == (N[0] + 4, N[1] + 4, 7) and np.array_equal(s[:, :, 0], a[:, :, 4])   # local k = -1 is global k = 3
    per = abi.make_params(*N, Re=100.0, dt=1e-3, bc={"Back": ("periodic",) * 3, "Front": ("periodic",) * 3})
    with pytest.raises(ValueError):
        zslab.slab_params(per, 0, 2, 5)


class NumpySlab:
    """GS.f90:35-68 on one slab in numpy (p-form, the oracle's operation
    order), behind the driver's backend interface."""

    def __init__(self, grid, gs, ge, state, dt, omega):
        import torch
        self.torch = torch
        self.gs, self.nz = gs, ge - gs + 1
        g = zslab.slab_grid(grid, gs, ge)
        P, US, VS, WS = (zslab.slab_halo(a, gs, ge).copy(order="F") for a in state)
        self.P, self.US, self.VS, self.WS = P, US, VS, WS
        self.dt, self.omega = dt, omega
        nx, ny, nz = P.shape[0] - 4, P.shape[1] - 4, self.nz
        c = slice(2, -2)
        self.iDx, self.Dxs = g["iDx"][c][:, None, None], g["Dxs"][c][:, None, None]
        self.Dxsm = g["Dxs"][1:-3][:, None, None]
        self.iDy, self.Dys = g["iDy"][c][None, :, None], g["Dys"][c][None, :, None]
        self.Dysm = g["Dys"][1:-3][None, :, None]
        self.iDz, self.Dzs = g["iDz"][c][None, None, :], g["Dzs"][c][None, None, :]
        self.Dzsm = g["Dzs"][1:-3][None, None, :]
        i, j, k = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1), np.arange(1, nz + 1), indexing="ij")
        self.parity = (i + j + k) & 1
        self.chmax = 0.0

    def plane_elems(self, field):
        return self.P.shape[0] * self.P.shape[1]

    def _arr(self, field):
        return self.WS if field == abi.FIELD_WSTAR else self.P

    def get(self, field, k0, count, comm):
        a = self._arr(field)[:, :, k0 + 1:k0 + 1 + count]
        return self.torch.from_numpy(np.ascontiguousarray(a.reshape(-1, order="F")))

    def put(self, field, k0, buf):
        a = self._arr(field)
        count = buf.numel() // self.plane_elems(field)
        a[:, :, k0 + 1:k0 + 1 + count] = buf.numpy().reshape(a.shape[0], a.shape[1], count, order="F")

    @staticmethod
    def sweep_field(colour):
        return abi.FIELD_P

    def stage(self, stage, colour=0):
        if stage == abi.STAGE_RHS:
            US, VS, WS, c = self.US, self.VS, self.WS, slice(2, -2)
            self.mc = ((US[c, c, c] - US[1:-3, c, c]) * self.iDy * self.iDz
                       + (VS[c, c, c] - VS[c, 1:-3, c]) * self.iDx * self.iDz
                       + (WS[c, c, c] - WS[c, c, 1:-3]) * self.iDx * self.iDy)
        elif stage == abi.STAGE_HALFSWEEP:
            P, c = self.P, slice(2, -2)
            iDx, iDy, iDz = self.iDx, self.iDy, self.iDz
            pc = P[c, c, c]
            pnew = (-P[3:-1, c, c] * iDy * iDz / self.Dxs
                    - P[1:-3, c, c] * iDy * iDz / self.Dxsm
                    - P[c, 3:-1, c] * iDx * iDz / self.Dys
                    - P[c, 1:-3, c] * iDx * iDz / self.Dysm
                    - P[c, c, 3:-1] * iDx * iDy / self.Dzs
                    - P[c, c, 1:-3] * iDx * iDy / self.Dzsm
                    + self.mc / self.dt) / (-iDy * iDz / self.Dxs - iDy * iDz / self.Dxsm
                                            - iDx * iDz / self.Dys - iDx * iDz / self.Dysm
                                            - iDx * iDy / self.Dzs - iDx * iDy / self.Dzsm)
            on = self.parity == colour
            ch = np.abs(pnew - pc)
            self.chmax = max(self.chmax, float(ch[on].max()))
            pc[on] = pc[on] + (self.omega * (pnew[on] - pc[on]))
        elif stage != abi.STAGE_CORRECT:
            raise AssertionError(stage)

    def change(self):
        x, self.chmax = self.chmax, 0.0
        return x


def _problem(orc):
    p = abi.make_params(*N, Re=100.0, dt=1e-3, zeta=1e-9, itmax=400, omega=1.6)
    grid = orc.gridder_unequal(*N, 1.0, 2.0, 3.0, (12.5, 0.7, 1.3, 2, 2, 3, 3, 5, 0.4, 0.5, 0.9, 0.8, 1.6))
    rng = np.random.default_rng(SEED)
    shape = [n + 4 for n in N]
    state = [np.asfortranarray(rng.standard_normal(shape)) for _ in range(4)]   # p, u*, v*, w*
    return p, grid, state


def _rank(rank, world, port, tmp):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from oracle import cpu_oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        p, grid, state = _problem(cpu_oracle)
        gs, ge, _ = zslab.partition(N[2], world)[rank]
        b = NumpySlab(grid, gs, ge, state, p.dt, p.omega)
        comm = zslab.SlabComm()
        run = zslab.SlabRun(b, comm, p)
        ik, conv, ch = run.sor_solve()
        np.savez(os.path.join(tmp, f"r{rank}.npz"), p=b.P[2:-2, 2:-2, 2:-2], ik=ik, conv=conv, ch=ch, gs=gs)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_sor_on_three_gloo_ranks_equals_the_single_domain_oracle(orc, tmp_path):
    world = 3
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_rank, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn")
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    # single domain: the oracle's red-black solve on the same inputs
    p, grid, state = _problem(orc)
    o = orc.Oracle(p, grid)
    for name, a in zip(("p", "u_star", "v_star", "w_star"), state):
        o.set(name, a)
    ik, _, conv = o.gauss_seidel()
    assert conv == 1
    ref = o.get("p")[2:-2, 2:-2, 2:-2]
    assert [int(r["gs"]) for r in parts] == [1, 5, 8]          # flips 0, 0, 1: both colour maps run
    assert 5 < ik < p.itmax
    for r in parts:
        assert int(r["ik"]) == ik and bool(r["conv"])
    got = np.concatenate([r["p"] for r in parts], axis=2)
    assert np.array_equal(got, ref)
