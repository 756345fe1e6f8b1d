"""The pressure operator of the reference's matrix assembly
(solver_1st_member.f90:19-29, written for its unused BiCGSTAB solver) against
the SOR operator of GS.f90:43-51 that the device runs, on a stretched grid.

* Interior rows: coef(ik,1) = sum of the six 1/(iD D*s) products and
  coef(ik,2..7) = -each of them, i.e. the GS.f90 coefficients a_nb =
  iDy iDz / Dxs, ... divided by the cell volume V = iDx iDy iDz.  These are
  the cE..cB tables of the device sweep.
* V times that operator is symmetric: V(i) cE(i) = V(i+1) cW(i+1) and so
  on.  The discrete adjoint solves its transposed pressure systems with the
  forward SOR through this identity (A^T y = l  <=>  A z = l / V, y = V z).
"""
import numpy as np

from ntustcfdlab_b200.solver import gridder_unequal

N = (9, 11, 13)
BAND = (12.5, 0.65, 0.6, 16, 4, 6, 4, 6, 1.0, 0.1, 0.3, 0.2, 0.5)


def metrics():
    g = gridder_unequal(*N, 1.0, 1.3, 1.7, BAND)
    F = lambda a: (lambda i: a[i + 1])        # index -1..n+2 stored from 0
    return {k: F(g[k]) for k in ("iDx", "Dxs", "iDy", "Dys", "iDz", "Dzs")}


def assembly(m):
    """solver_1st_member.f90:19-29, interior rows (before the boundary edits of 32-66)."""
    nx, ny, nz = N
    coef = np.zeros((nx * ny * nz, 7))
    ik = 0
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                e = 1 / m["iDx"](i) / m["Dxs"](i)
                w = 1 / m["iDx"](i) / m["Dxs"](i - 1)
                n = 1 / m["iDy"](j) / m["Dys"](j)
                s = 1 / m["iDy"](j) / m["Dys"](j - 1)
                f = 1 / m["iDz"](k) / m["Dzs"](k)
                b = 1 / m["iDz"](k) / m["Dzs"](k - 1)
                coef[ik] = (e + w + n + s + f + b, -e, -w, -n, -s, -f, -b)
                ik += 1
    return coef


def test_assembly_is_the_sor_operator_over_the_volume():
    m = metrics()
    coef = assembly(m)
    nx, ny, nz = N
    ik = 0
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                V = m["iDx"](i) * m["iDy"](j) * m["iDz"](k)
                # GS.f90:43-51 coefficients
                a = (m["iDy"](j) * m["iDz"](k) / m["Dxs"](i), m["iDy"](j) * m["iDz"](k) / m["Dxs"](i - 1),
                     m["iDx"](i) * m["iDz"](k) / m["Dys"](j), m["iDx"](i) * m["iDz"](k) / m["Dys"](j - 1),
                     m["iDx"](i) * m["iDy"](j) / m["Dzs"](k), m["iDx"](i) * m["iDy"](j) / m["Dzs"](k - 1))
                np.testing.assert_allclose(-coef[ik, 1:], np.array(a) / V, rtol=1e-14)
                np.testing.assert_allclose(coef[ik, 0], sum(a) / V, rtol=1e-14)
                ik += 1


def test_volume_weighted_operator_is_symmetric():
    m = metrics()
    coef = assembly(m)
    nx, ny, nz = N
    V = lambda i, j, k: m["iDx"](i) * m["iDy"](j) * m["iDz"](k)
    row = lambda i, j, k: (i - 1) + nx * ((j - 1) + ny * (k - 1))
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                r = row(i, j, k)
                if i < nx:
                    np.testing.assert_allclose(V(i, j, k) * coef[r, 1], V(i + 1, j, k) * coef[row(i + 1, j, k), 2],
                                               rtol=1e-13)
                if j < ny:
                    np.testing.assert_allclose(V(i, j, k) * coef[r, 3], V(i, j + 1, k) * coef[row(i, j + 1, k), 4],
                                               rtol=1e-13)
                if k < nz:
                    np.testing.assert_allclose(V(i, j, k) * coef[r, 5], V(i, j, k + 1) * coef[row(i, j, k + 1), 6],
                                               rtol=1e-13)
