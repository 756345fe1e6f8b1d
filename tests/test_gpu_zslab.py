"""z-slab decomposition through the CUDA library (ntcfd_slab_stage): one
slab equals ntcfd_step, and three slabs -- three processes on this GPU that
exchange their planes through the host (gloo), so no kernel of one waits on
another's -- equal the single-domain FP64 step bit for bit over several
steps with LES, a body, an inflow wall and a Neumann outflow."""
import ctypes
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from ntustcfdlab_b200 import abi, zslab  # noqa: E402

pytestmark = pytest.mark.gpu

N = (16, 12, 10)          # over 3 ranks: planes 1-4, 5-7, 8-10 (the last slab's colours flip)
STEPS = 4
SEED = 7


def _params():
    bc = {"West": ("periodic",) * 3, "East": ("periodic",) * 3,
          "South": ("Neumann",) * 3, "North": ("Neumann",) * 3,
          "Back": ("Dirichlet", "Dirichlet", "Dirichlet"), "Front": ("Neumann",) * 3}
    return abi.make_params(*N, Re=500.0, dt=abi.f4(2e-3), LES=1, smag_mode=abi.SMAG_STAGGERED, bc=bc,
                           bc_value={"Back": (0.0, 0.0, 1.0)}, sor_path=abi.SOR_STREAMING, zeta=1e-8)


def _grid():
    from ntustcfdlab_b200.solver import gridder_unequal
    return gridder_unequal(*N, 1.0, 3.0, 4.0, (12.5, 1.2, 1.6, 4, 4, 8, 3, 6, 1.0, 0.4, 1.2, 0.6, 1.2))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _single_domain(tmp):
    """Initial state (after the BCs) and the single-domain result."""
    from ntustcfdlab_b200.solver import Solver
    s = Solver(_params(), _grid())
    try:
        rng = np.random.default_rng(SEED)
        shape = s.halo_shape
        s.set_state(*[np.asfortranarray(0.1 * rng.standard_normal(shape)) for _ in range(3)],
                    np.zeros(shape, order="F"))
        s.build_mask_cylinder(2.0, 1.5, 0.4)
        s.boundary_conditions()
        init, eta = s.get_state(), s.get_mask()
        np.savez(os.path.join(tmp, "init.npz"), u=init[0], v=init[1], w=init[2], p=init[3], eta=eta)
        info, _ = s.step(STEPS)
        return s.get_state(), [i.sor_iters for i in info]
    finally:
        s.close()


def _run_slabs(rank, world, tmp):
    comm = zslab.SlabComm()
    d = np.load(os.path.join(tmp, "init.npz"))
    b = zslab.LibrarySlab(_params(), _grid(), rank, world)
    try:
        b.solver.set_state(*[zslab.slab_halo(d[k], b.gs, b.ge) for k in "uvwp"])
        b.solver.set_mask(zslab.slab_halo(d["eta"], b.gs, b.ge))
        run = zslab.SlabRun(b, comm, _params())
        sweeps = [run.step()[0] for _ in range(STEPS)]
        st = b.solver.get_state()
        np.savez(os.path.join(tmp, f"r{rank}.npz"), sweeps=sweeps, gs=b.gs, time=b.solver.time,
                 **{k: a[2:-2, 2:-2, 2:-2] for k, a in zip("uvwp", st)})
    finally:
        b.close()


def _rank(rank, world, port, tmp):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        _run_slabs(rank, world, tmp)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("world", [1, 3])
def test_slabs_repeat_the_single_domain_step(tmp_path, world):
    ref, ref_sweeps = _single_domain(str(tmp_path))
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    assert [int(r["gs"]) for r in parts] == [g for g, _, _ in zslab.partition(N[2], world)]
    for r in parts:
        assert list(r["sweeps"]) == ref_sweeps
        assert float(r["time"]) > 0
    assert min(ref_sweeps) > 3
    for k, a in zip("uvwp", ref):
        got = np.concatenate([r[k] for r in parts], axis=2)
        assert np.array_equal(got, a[2:-2, 2:-2, 2:-2]), k


def test_slab_contexts_refuse_ntcfd_step_mixed_precision_and_the_aliased_smagorinsky():
    from ntustcfdlab_b200.solver import NtcfdError, Solver
    p = zslab.slab_params(_params(), 1, 3, 3)
    s = Solver(p, zslab.slab_grid(_grid(), 5, 7))
    try:
        with pytest.raises(NtcfdError, match="ntcfd_slab_stage"):
            s.step(1)
        assert s.lib.ntcfd_slab_stage(s.h, 99, 0) == abi.NTCFD_EINVAL
        buf = np.zeros(4 * s.lib.ntcfd_slab_plane_elems(s.h, abi.FIELD_U))
        assert s.lib.ntcfd_slab_planes(s.h, abi.FIELD_U, 2, 4, buf.ctypes.data_as(ctypes.c_void_p), 0) == 0
        assert s.lib.ntcfd_slab_planes(s.h, abi.FIELD_U, 3, 4, buf.ctypes.data_as(ctypes.c_void_p), 0) \
            == abi.NTCFD_EINVAL                      # planes 3..6: past nz + 2 = 5
    finally:
        s.close()
    for change in (dict(precision=abi.MIXED), dict(smag_mode=abi.SMAG_REF_ALIASED)):
        m = Solver(abi.params_copy(p, **change), zslab.slab_grid(_grid(), 5, 7))
        try:
            assert m.lib.ntcfd_slab_stage(m.h, abi.STAGE_PREDICT, 0) == abi.NTCFD_EINVAL
        finally:
            m.close()
