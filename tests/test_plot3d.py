"""PLOT3D files in the reference's format (gridder.f90:150-212,
filer.f90:161-187, reading_data.f90:62-90), checked byte for byte against a
numpy reading of Fortran unformatted sequential records (4-byte length,
payload, 4-byte length; default reals are float32)."""
import numpy as np

from ntustcfdlab_b200.abi import dptr
from ntustcfdlab_b200.solver import gridder_unequal, read_plot3d_q, write_plot3d_q, write_plot3d_x

NX, NY, NZ = 6, 5, 4


def records(path):
    raw = open(path, "rb").read()
    out, q = [], 0
    while q < len(raw):
        n = int(np.frombuffer(raw, "<i4", 1, q)[0])
        out.append(raw[q + 4:q + 4 + n])
        assert int(np.frombuffer(raw, "<i4", 1, q + 4 + n)[0]) == n
        q += 8 + n
    return out


def grid():
    band = (12.5, 2.0, 2.0, 2, 2, 3, 2, 3, 1.0, 0.3, 0.6, 1.1, 2.0)
    return gridder_unequal(NX, NY, NZ, 1.0, 4.0, 4.0, band)


def fields(seed=5):
    rng = np.random.default_rng(seed)
    inner = [np.asfortranarray(rng.standard_normal((NX, NY, NZ))) for _ in range(4)]
    eta = np.asfortranarray(rng.random((NX + 4, NY + 4, NZ + 4)))
    return inner, eta


def test_grid_file_holds_cell_centres(ntcfd_lib, tmp_path):
    g = grid()
    path = str(tmp_path / "mesh.x")
    write_plot3d_x(path, g)
    r = records(path)
    assert len(r) == 3
    assert np.frombuffer(r[0], "<i4").tolist() == [1]
    assert np.frombuffer(r[1], "<i4").tolist() == [NX, NY, NZ]
    xyz = np.frombuffer(r[2], "<f4").reshape(3, NZ, NY, NX)   # C view of (nx,ny,nz) Fortran blocks
    # X(i) sits at index i + 1 (index -1..n+3); centres (X(i+1) + X(i)) / 2 for i = 1..n
    centres = [((g[a][3:-2] + g[a][2:-3]) / 2.0).astype(np.float32) for a in "XYZ"]
    for a, (axis, c) in enumerate(zip("XYZ", centres)):
        shape = [1, 1, 1]
        shape[2 - a] = -1
        want = np.broadcast_to(c.reshape(shape), (NZ, NY, NX))
        assert np.array_equal(xyz[a], want), axis


def test_solution_file_layout_and_append(ntcfd_lib, tmp_path):
    (pre, uc, vc, wc), eta = fields()
    path = str(tmp_path / "0000.q")
    write_plot3d_q(path, pre, uc, vc, wc, eta, append=False)
    write_plot3d_q(path, 2 * pre, uc, vc, wc, eta)      # the reference appends
    r = records(path)
    assert len(r) == 8
    for b in (0, 4):
        assert np.frombuffer(r[b], "<i4").tolist() == [1]
        assert np.frombuffer(r[b + 1], "<i4").tolist() == [NX, NY, NZ]
        assert np.frombuffer(r[b + 2], "<f4").tolist() == [1.0] * 4
    q = np.frombuffer(r[3], "<f4").reshape(5, NX * NY * NZ)
    for h, a in enumerate((pre, uc, vc, wc, eta[2:-2, 2:-2, 2:-2])):
        assert np.array_equal(q[h], a.ravel(order="F").astype(np.float32))
    q2 = np.frombuffer(r[7], "<f4").reshape(5, NX * NY * NZ)
    assert np.array_equal(q2[0], (2 * pre).ravel(order="F").astype(np.float32))


def test_restart_reconstructs_faces_like_the_reference(ntcfd_lib, tmp_path):
    (pre, uc, vc, wc), eta = fields(9)
    path = str(tmp_path / "in.q")
    write_plot3d_q(path, pre, uc, vc, wc, eta, append=False)
    shape = (NX + 4, NY + 4, NZ + 4)
    u, v, w, p = (np.full(shape, 7.0, order="F") for _ in range(4))
    read_plot3d_q(path, u, v, w, p)
    f = [a.astype(np.float32) for a in (pre, uc, vc, wc)]
    half = np.float32(0.5)
    # faces on 1..n-1 in every direction, default-real arithmetic; array index = Fortran + 1
    want_u = (half * (f[1][0:NX - 1, 0:NY - 1, 0:NZ - 1] + f[1][1:NX, 0:NY - 1, 0:NZ - 1])).astype(np.float64)
    want_v = (half * (f[2][0:NX - 1, 0:NY - 1, 0:NZ - 1] + f[2][0:NX - 1, 1:NY, 0:NZ - 1])).astype(np.float64)
    want_w = (half * (f[3][0:NX - 1, 0:NY - 1, 0:NZ - 1] + f[3][0:NX - 1, 0:NY - 1, 1:NZ])).astype(np.float64)
    inner = np.s_[2:NX + 1, 2:NY + 1, 2:NZ + 1]
    assert np.array_equal(u[inner], want_u)
    assert np.array_equal(v[inner], want_v)
    assert np.array_equal(w[inner], want_w)
    assert np.array_equal(p[2:-2, 2:-2, 2:-2], f[0].astype(np.float64))
    # everything else keeps the caller's values
    for a in (u, v, w):
        m = np.ones(shape, bool)
        m[inner] = False
        assert np.all(a[m] == 7.0)
    m = np.ones(shape, bool)
    m[2:-2, 2:-2, 2:-2] = False
    assert np.all(p[m] == 7.0)


def test_restart_rejects_a_file_of_another_grid(ntcfd_lib, tmp_path):
    (pre, uc, vc, wc), eta = fields()
    path = str(tmp_path / "in.q")
    write_plot3d_q(path, pre, uc, vc, wc, eta, append=False)
    u = np.zeros((NX + 5, NY + 4, NZ + 4), order="F")
    assert ntcfd_lib.ntcfd_read_plot3d_q(path.encode(), NX + 1, NY, NZ, *[dptr(u)] * 4) == -3
