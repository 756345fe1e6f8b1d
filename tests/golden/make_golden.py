"""Generates the committed fixtures of tests/golden.

    python tests/golden/make_golden.py --reference <checkout of the reference>

naca_dat.npz      every 10th point (and the closing point) of the reference's
                  airfoil files NACA0012.DAT and NACA0015.DAT, which
                  airfoil.f90:580-600 reads as the RayCasting polygon.  Only
                  this script reads the reference tree; the tests read the
                  committed subset.
oracle_*.npz      outputs of the CPU oracle (oracle/, single thread) on small
                  cases: a cavity after 3 steps (red-black and lexicographic
                  SOR), an LES step on a stretched grid with a cylinder, the
                  cylinder mask, and the ray-cast mask of the NACA0012.DAT
                  subset.  They freeze the oracle so that a later change to
                  it, or to the device path, shows up as a fixture mismatch.
oracle_schemes.npz the uncalled predictors discretisation_QUICK.f90,
                  _upwind.f90 and _centre.f90: per scheme a cavity after 3
                  steps and two LES steps with a cylinder (interior values).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ntustcfdlab_b200.abi import (CENTRE, QUICK, SOR_LEX, SOR_REDBLACK, SMAG_REF_ALIASED,  # noqa: E402
                                  UPWIND, f4, make_params)
from oracle import cpu_oracle  # noqa: E402

DECIMATE = 10

# small cases shared with tests/test_golden.py and tests/test_gpu_golden.py
CAVITY = dict(n=(12, 10, 8), Re=100.0, dt=f4(1e-3), steps=3)
LES = dict(n=(8, 24, 32), L=(1.0, 6.0, 8.0), Re=1000.0, dt=0.01, Cs=f4(0.18), forced=7, seed=3,
           cyl=(2.55, 3.1, 0.5))
NACA_GRID = dict(n=(4, 48, 64), L=(1.0, 3.0, 4.0),
                 band=(f4(12.5), 1.5, 1.2, 4, 20, 30, 24, 36, 1.0, f4(0.3), f4(0.6), f4(1.1), 2.0),
                 aoa=5.0, zc=1.2, yc=1.5)


SCHEMES = ((QUICK, "quick"), (UPWIND, "upwind"), (CENTRE, "centre"))
SCHEME_LES = dict(n=(6, 12, 16), L=(1.0, 3.0, 4.0), forced=(5, 5), seed=11, cyl=(2.05, 1.55, 0.5))


def cavity_params(sor, scheme=0):
    n = CAVITY["n"]
    return make_params(*n, Re=CAVITY["Re"], dt=CAVITY["dt"], sor_order=sor, scheme=scheme,
                       bc={"North": ("Dirichlet", "no-slip", "no-slip")})


def les_params():
    n = LES["n"]
    bc = {"West": ("periodic",) * 3, "East": ("periodic",) * 3,
          "South": ("Neumann",) * 3, "North": ("Neumann",) * 3,
          "Back": ("Dirichlet", "Dirichlet", "Dirichlet"), "Front": ("Neumann",) * 3}
    return make_params(*n, Re=LES["Re"], dt=LES["dt"], LES=1, Cs=LES["Cs"], smag_mode=SMAG_REF_ALIASED,
                       bc=bc, bc_value={"Back": (0.0, 0.1, 1.0)}, lx=LES["L"][0])


def scheme_les_params(scheme):
    c = SCHEME_LES
    bc = {"West": ("periodic",) * 3, "East": ("periodic",) * 3,
          "South": ("Neumann",) * 3, "North": ("Neumann",) * 3,
          "Back": ("Dirichlet", "Dirichlet", "Dirichlet"), "Front": ("Neumann",) * 3}
    return make_params(*c["n"], Re=LES["Re"], dt=LES["dt"], LES=1, Cs=LES["Cs"], scheme=scheme,
                       bc=bc, bc_value={"Back": (0.0, 0.1, 1.0)}, lx=c["L"][0])


def les_state(seed=None, n=None):
    n = n or LES["n"]
    shape = (n[0] + 4, n[1] + 4, n[2] + 4)
    rng = np.random.default_rng(LES["seed"] if seed is None else seed)
    u = 0.05 * rng.standard_normal(shape)
    v = 0.1 + 0.05 * rng.standard_normal(shape)
    w = 1.0 + 0.05 * rng.standard_normal(shape)
    p = 0.01 * rng.standard_normal(shape)
    return [np.asfortranarray(a) for a in (u, v, w, p)]


def oracle_cavity(sor):
    o = cpu_oracle.Oracle(cavity_params(sor), cpu_oracle.gridder_equal(*CAVITY["n"], 1.0, 1.0, 1.0))
    o.initial_conditions()
    o.boundary_conditions()
    info = o.step(CAVITY["steps"])
    return {k: o.get(k) for k in ("u", "v", "w", "p")}, np.array([i.sor_iters for i in info])


def oracle_les_step():
    n, L = LES["n"], LES["L"]
    o = cpu_oracle.Oracle(les_params(), cpu_oracle.gridder_equal(*n, *L))
    o.initial_conditions()
    zc, yc, r = LES["cyl"]
    o.cylinder(zc, yc, r)
    for k, a in zip("uvwp", les_state()):
        o.set(k, a)
    o.boundary_conditions()
    info = o.step(1, forced=[LES["forced"]])
    out = {k: o.get(k) for k in ("u", "v", "w", "p", "ETA")}
    out["cdrag"] = np.array([info[0].cDrag])
    out["clift"] = np.array([info[0].cLift])
    return out


def inner(a):
    return np.asfortranarray(a[2:-2, 2:-2, 2:-2])


def oracle_schemes():
    out = {}
    c = SCHEME_LES
    for scheme, tag in SCHEMES:
        o = cpu_oracle.Oracle(cavity_params(SOR_REDBLACK, scheme),
                              cpu_oracle.gridder_equal(*CAVITY["n"], 1.0, 1.0, 1.0))
        o.initial_conditions()
        o.boundary_conditions()
        info = o.step(CAVITY["steps"])
        for k in "uvwp":
            out[f"{tag}_cavity_{k}"] = inner(o.get(k))
        out[f"{tag}_cavity_sweeps"] = np.array([i.sor_iters for i in info])
        o = cpu_oracle.Oracle(scheme_les_params(scheme), cpu_oracle.gridder_equal(*c["n"], *c["L"]))
        o.initial_conditions()
        o.cylinder(*c["cyl"])
        for k, a in zip("uvwp", les_state(c["seed"], c["n"])):
            o.set(k, a)
        o.boundary_conditions()
        o.step(len(c["forced"]), forced=list(c["forced"]))
        for k in "uvwp":
            out[f"{tag}_les_{k}"] = inner(o.get(k))
    return out


def oracle_naca_mask(az, ay):
    g = NACA_GRID
    p = make_params(*g["n"], Re=100.0, dt=f4(1e-3))
    o = cpu_oracle.Oracle(p, cpu_oracle.gridder_unequal(*g["n"], *g["L"], g["band"]))
    o.initial_conditions()
    ties = o.raycasting(az, ay, g["aoa"], g["zc"], g["yc"])
    return o.get("ETA"), ties


def read_dat(path):
    d = np.loadtxt(path)
    keep = list(range(0, len(d), DECIMATE))
    if keep[-1] != len(d) - 1:
        keep.append(len(d) - 1)
    return d[keep]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="directory of the reference checkout (holds NACA0012.DAT, NACA0015.DAT)")
    args = ap.parse_args()
    cpu_oracle.build()
    d12 = read_dat(os.path.join(args.reference, "NACA0012.DAT"))
    d15 = read_dat(os.path.join(args.reference, "NACA0015.DAT"))
    np.savez_compressed(os.path.join(HERE, "naca_dat.npz"), naca0012=d12, naca0015=d15,
                        decimate=np.array([DECIMATE]))
    for sor, tag in ((SOR_REDBLACK, "redblack"), (SOR_LEX, "lex")):
        f, sweeps = oracle_cavity(sor)
        np.savez_compressed(os.path.join(HERE, f"oracle_cavity_{tag}.npz"), sweeps=sweeps, **f)
    np.savez_compressed(os.path.join(HERE, "oracle_les_cylinder.npz"), **oracle_les_step())
    np.savez_compressed(os.path.join(HERE, "oracle_schemes.npz"), **oracle_schemes())
    eta, ties = oracle_naca_mask(np.ascontiguousarray(d12[:, 0]), np.ascontiguousarray(d12[:, 1]))
    np.savez_compressed(os.path.join(HERE, "oracle_naca0012_dat_mask.npz"), ETA=eta, ties=np.array([ties]))
    for fn in sorted(os.listdir(HERE)):
        if fn.endswith(".npz"):
            print(f"{fn:36s} {os.path.getsize(os.path.join(HERE, fn)):8d} bytes")


if __name__ == "__main__":
    main()
