"""The device path against the committed oracle fixtures of tests/golden
(the fixtures are the oracle's outputs; see tests/golden/make_golden.py)."""
import importlib.util
import os

import numpy as np
import pytest

from conftest import interior, rel_l2
from ntustcfdlab_b200.abi import params_copy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _mg():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _load(name):
    return np.load(os.path.join(GOLD, name))


def test_cavity_steps_match_fixture():
    from ntustcfdlab_b200.solver import Solver, gridder_equal
    mg = _mg()
    g = _load("oracle_cavity_redblack.npz")
    p = mg.cavity_params(mg.SOR_REDBLACK)
    s = Solver(p, gridder_equal(*mg.CAVITY["n"], 1.0, 1.0, 1.0))
    try:
        s.boundary_conditions()
        info, rc = s.step(mg.CAVITY["steps"])
        assert [i.sor_iters for i in info] == list(g["sweeps"])
        for k, a in zip("uvwp", s.get_state()):
            assert rel_l2(interior(a), interior(g[k])) <= 1e-12, k
    finally:
        s.close()


def test_les_cylinder_step_matches_fixture():
    from ntustcfdlab_b200.solver import Solver, gridder_equal
    mg = _mg()
    g = _load("oracle_les_cylinder.npz")
    p = params_copy(mg.les_params(), zeta=0.0, itmax=mg.LES["forced"])
    s = Solver(p, gridder_equal(*mg.LES["n"], *mg.LES["L"]))
    try:
        s.build_mask_cylinder(*mg.LES["cyl"])
        assert np.array_equal(s.get_mask(), g["ETA"])
        s.set_state(*mg.les_state())
        s.boundary_conditions()
        info, rc = s.step(1)
        for k, a in zip("uvwp", s.get_state()):
            assert rel_l2(interior(a), interior(g[k])) <= 1e-12, k
        assert abs(info[0].cDrag - g["cdrag"][0]) <= 1e-10 * abs(g["cdrag"][0])
        assert abs(info[0].cLift - g["clift"][0]) <= 1e-10 * abs(g["clift"][0])
    finally:
        s.close()


def test_raycasting_of_reference_points_matches_fixture():
    from ntustcfdlab_b200.abi import f4, make_params
    from ntustcfdlab_b200.solver import Solver, gridder_unequal
    mg = _mg()
    g = _load("oracle_naca0012_dat_mask.npz")
    d = _load("naca_dat.npz")["naca0012"]
    G = mg.NACA_GRID
    s = Solver(make_params(*G["n"], Re=100.0, dt=f4(1e-3)), gridder_unequal(*G["n"], *G["L"], G["band"]))
    try:
        ties = s.build_mask_polygon(d[:, 0], d[:, 1], G["aoa"], G["zc"], G["yc"])
        assert ties == int(g["ties"][0])
        assert np.array_equal(s.get_mask(), g["ETA"])
    finally:
        s.close()
