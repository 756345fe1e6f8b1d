"""GPU parity of the uncalled K2 predictors (discretisation_QUICK.f90,
discretisation_upwind.f90, discretisation_centre.f90) against the oracle.

The device evaluates the reference's algebra with tabulated reciprocals, so
FP64 fields agree to rounding: relative L2 <= 1e-12 per field after the
same forced sweep counts, and identical sweep counts where the stop rule
runs.  The wall faces that the schemes do not predict must keep u exactly.
"""
import importlib.util
import os

import numpy as np
import pytest

from conftest import interior, rel_l2
from ntustcfdlab_b200.abi import (CENTRE, MIXED, QUICK, SOR_RESIDENT, SOR_STREAMING, UPWIND, f4, make_params,
                                  params_copy)

pytestmark = pytest.mark.gpu

SCHEMES = {"quick": QUICK, "upwind": UPWIND, "centre": CENTRE}
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
BAND = (12.5, 0.65, 0.6, 16, 4, 6, 4, 6, 1.0, 0.1, 0.3, 0.2, 0.5)
BCS = {"West": ("no-slip", "Neumann", "Dirichlet"), "East": ("Neumann", "no-slip", "Neumann"),
       "South": ("Neumann", "no-slip", "Dirichlet"), "North": ("Dirichlet", "Neumann", "no-slip"),
       "Back": ("Dirichlet", "Neumann", "Dirichlet"), "Front": ("Neumann", "Neumann", "Neumann")}


def _mg():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _pair(orc, p, grid, state):
    from ntustcfdlab_b200.solver import Solver
    s = Solver(p, grid)
    o = orc.Oracle(p, grid)
    o.initial_conditions()
    s.set_state(*state)
    for k, a in zip("uvwp", state):
        o.set(k, a)
    s.boundary_conditions()
    o.boundary_conditions()
    return s, o


@pytest.mark.parametrize("les", [0, 1])
@pytest.mark.parametrize("path", [SOR_STREAMING, SOR_RESIDENT])
@pytest.mark.parametrize("name", list(SCHEMES))
def test_forced_steps_on_a_stretched_grid(orc, name, path, les):
    n = (13, 11, 9)
    g = orc.gridder_unequal(*n, 1.0, 1.3, 1.7, BAND)
    p = make_params(*n, Re=100.0, dt=f4(1e-3), zeta=0.0, itmax=6, bc=BCS, LES=les, Cs=f4(0.18),
                    bc_value={"Back": (0.3, -0.2, 1.0)}, sor_path=path, scheme=SCHEMES[name])
    rng = np.random.default_rng(21)
    state = [np.asfortranarray(0.3 * rng.standard_normal((17, 15, 13))) for _ in range(4)]
    s, o = _pair(orc, p, g, state)
    try:
        s.step(2)
        o.step(2, forced=[6, 6])
        got = s.get_state()
        for k, a in zip("uvwp", got):
            assert rel_l2(interior(a), interior(o.get(k))) <= 1e-12, k
    finally:
        s.close()


@pytest.mark.parametrize("name", list(SCHEMES))
def test_fixture_cavity_and_les(name):
    """The committed oracle outputs of tests/golden/oracle_schemes.npz."""
    from ntustcfdlab_b200.solver import Solver, gridder_equal
    mg = _mg()
    g = np.load(os.path.join(GOLD, "oracle_schemes.npz"))
    scheme = SCHEMES[name]
    s = Solver(mg.cavity_params(mg.SOR_REDBLACK, scheme), gridder_equal(*mg.CAVITY["n"], 1.0, 1.0, 1.0))
    try:
        s.boundary_conditions()
        info, rc = s.step(mg.CAVITY["steps"])
        assert [i.sor_iters for i in info] == list(g[f"{name}_cavity_sweeps"])
        for k, a in zip("uvwp", s.get_state()):
            assert rel_l2(interior(a), g[f"{name}_cavity_{k}"]) <= 1e-12, k
    finally:
        s.close()
    c = mg.SCHEME_LES
    forced = c["forced"]
    p = params_copy(mg.scheme_les_params(scheme), zeta=0.0, itmax=forced[0])
    s = Solver(p, gridder_equal(*c["n"], *c["L"]))
    try:
        s.build_mask_cylinder(*c["cyl"])
        s.set_state(*mg.les_state(c["seed"], c["n"]))
        s.boundary_conditions()
        s.step(len(forced))
        for k, a in zip("uvwp", s.get_state()):
            assert rel_l2(interior(a), g[f"{name}_les_{k}"]) <= 1e-12, k
    finally:
        s.close()


@pytest.mark.parametrize("name", list(SCHEMES))
def test_mixed_precision_converged_steps(orc, name):
    """The mixed path with the stop rule running: same sweep counts as the
    FP64 oracle within one sweep, fields within the mixed tolerance."""
    from ntustcfdlab_b200 import cases
    c = cases.cavity(24, 400.0, 1e-3, 10)
    p = params_copy(c.params, scheme=SCHEMES[name])
    shape = (28, 28, 28)
    zero = [np.zeros(shape, order="F") for _ in range(4)]
    res = {}
    for prec in (0, MIXED):
        s, o = _pair(orc, params_copy(p, precision=prec, mixed_cycle=8), c.grid, zero)
        try:
            info, rc = s.step(c.steps)
            res[prec] = (s.get_state(), [i.sor_iters for i in info])
            if prec == 0:
                oi = o.step(c.steps)
                assert [i.sor_iters for i in info] == [i.sor_iters for i in oi]
                for k, a in zip("uvwp", res[prec][0]):
                    assert rel_l2(interior(a), interior(o.get(k))) <= 1e-11, k
        finally:
            s.close()
    for k, a, b in zip("uvwp", res[0][0], res[MIXED][0]):
        assert rel_l2(interior(b), interior(a)) <= 1e-6, k


def test_adjoint_refuses_other_schemes():
    from ntustcfdlab_b200 import cases
    from ntustcfdlab_b200.solver import NtcfdError, Solver
    c = cases.cavity(12, 100.0, 1e-3, 2)
    s = Solver(params_copy(c.params, scheme=UPWIND), c.grid)
    try:
        s.boundary_conditions()
        with pytest.raises(NtcfdError):
            s.adjoint(2, 1)
        s.step(1)
    finally:
        s.close()
