"""Diagnostics series, fluctuation field and Q-criterion: the oracle against
known answers and the file formats (CPU only)."""
import math

import numpy as np

from compchan3dmpi_b200.mesh import periodic_coords, mesh_cosine
from compchan3dmpi_b200.stats import append_diag_series, write_q_invariant
from oracle import oracle as O


def _field(n1, n2, n3, rho=1.3, u=0.7, v=-0.2, w=0.1):
    var = np.zeros((7, n3, n2, n1))
    var[0] = rho; var[1] = u; var[2] = v; var[3] = w
    var[5] = 1.0; var[4] = 2.0; var[6] = 0.5
    return var


def test_uniform_field_known_answers():
    n1, n2, n3 = 16, 10, 13
    x3, _, _ = mesh_cosine(n3)
    Ly = 4 * math.pi / 3
    dy = Ly / (n2 - 1)
    x2end = periodic_coords(n2, Ly)[-1]
    planes = [5, 10, 2, 14, 3, 70]
    out = O.diagnostics(_field(n1, n2, n3), planes, x3, dy, x2end)
    assert math.isclose(out[0], 0.7 ** 2 + 0.2 ** 2 + 0.1 ** 2, rel_tol=1e-12)  # sequential sum of N terms
    np_ = len(planes)
    rho_b, u_b, m_b = out[1:1 + np_], out[1 + np_:1 + 2 * np_], out[1 + 2 * np_:]
    inside = np.array([3 <= p <= n1 - 2 for p in planes])
    # the cell heights telescope to x3(nP3) - x3(1) = x3(nP3); dy*(nP2-1) = x2(nP2) up to rounding
    assert np.allclose(rho_b[inside], 1.3, rtol=1e-13) and np.all(rho_b[~inside] == 0)
    assert np.allclose(u_b[inside], 0.7, rtol=1e-13) and np.all(u_b[~inside] == 0)
    assert np.allclose(m_b[inside], 1.3 * 0.7, rtol=1e-13) and np.all(m_b[~inside] == 0)


def test_plane_quadrature_matches_trapezoid():
    rng = np.random.default_rng(7)
    n1, n2, n3 = 12, 9, 11
    var = rng.uniform(0.5, 1.5, size=(7, n3, n2, n1))
    x3, _, _ = mesh_cosine(n3)
    dy = 0.3
    out = O.diagnostics(var, [4], x3, dy, 2.5)
    f = var[0][:, :, 3]                                      # plane i=4: (k, j)
    cell = 0.25 * (f[:-1, :-1] + f[:-1, 1:] + f[1:, :-1] + f[1:, 1:])
    want = np.sum(cell * (dy * np.diff(x3))[:, None]) / (x3[-1] * 2.5)
    assert math.isclose(out[1], want, rel_tol=1e-13)
    fm = var[0][:, :, 3] * var[1][:, :, 3]
    cell = 0.25 * (fm[:-1, :-1] + fm[:-1, 1:] + fm[1:, :-1] + fm[1:, 1:])
    assert math.isclose(out[3], np.sum(cell * (dy * np.diff(x3))[:, None]) / (x3[-1] * 2.5), rel_tol=1e-13)


def _grid(n1=9, n2=8, n3=7, seed=3):
    rng = np.random.default_rng(seed)
    x = np.cumsum(np.r_[0, rng.uniform(0.5, 1.5, n1 - 1)])
    y = np.cumsum(np.r_[0, rng.uniform(0.5, 1.5, n2 - 1)])
    z = np.cumsum(np.r_[0, rng.uniform(0.5, 1.5, n3 - 1)])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return x, y, z, X, Y, Z


def test_q_criterion_known_answers():
    x, y, z, X, Y, Z = _grid()
    inner = (slice(1, -1),) * 3
    om = 1.7
    Q = O.qcrit(-om * Y, om * X, 0 * X, x, y, z)          # solid-body rotation: Q = omega^2
    assert np.allclose(Q[inner], om ** 2, rtol=1e-13)
    assert np.all(Q[0] == 0) and np.all(Q[:, :, -1] == 0)
    a = 0.8
    Q = O.qcrit(a * X, -a * Y, 0 * X, x, y, z)             # plane strain: Q = -a^2
    assert np.allclose(Q[inner], -a * a, rtol=1e-13)
    # Q of a linear field is -1/2 tr(J^2) + 1/2 tr(J)^2 - ... : general check
    J = np.array([[0.3, -1.1, 0.4], [0.9, -0.2, 0.5], [-0.6, 0.7, 0.1]])
    U = [J[c, 0] * X + J[c, 1] * Y + J[c, 2] * Z for c in range(3)]
    Q = O.qcrit(*U, x, y, z)
    S = 0.5 * (J + J.T); R = 0.5 * (J - J.T)
    want = 0.5 * (np.trace(J) ** 2 - np.sum(S * S) + np.sum(R * R))
    assert np.allclose(Q[inner], want, rtol=1e-12, atol=1e-13)


def test_fluctuation_is_plane_mean_removal():
    rng = np.random.default_rng(1)
    var = rng.normal(size=(7, 5, 4, 3))
    mean = rng.normal(size=(7, 5))
    f = O.fluctuation(var, mean)
    assert np.array_equal(f[:, 2, 1, 0], var[:, 2, 1, 0] - mean[:, 2])


def test_series_and_q_file_formats(tmp_path):
    d = {"time": np.array([0.001, 0.002]), "ke": np.array([0.25, 0.5]),
         "rho_b": np.ones((2, 5)), "u_b": np.full((2, 5), 0.5), "rhou_b": np.full((2, 5), -0.5)}
    append_diag_series(tmp_path, d)
    append_diag_series(tmp_path, d)
    ke = (tmp_path / "KE.dat").read_text().splitlines()
    assert len(ke) == 4 and ke[0] == "       0.0010000       0.2500000"
    m = (tmp_path / "massflow.dat").read_text().splitlines()[0]
    assert len(m) == 6 * 16 and m.split()[1] == "-0.5000000"
    Q = np.arange(2 * 3 * 4, dtype=float).reshape(2, 3, 4)
    write_q_invariant(tmp_path / "q.dat", np.arange(4.0), np.arange(3.0), np.arange(2.0), Q)
    lines = (tmp_path / "q.dat").read_text().splitlines()
    assert lines[2] == 'ZONE i=  4,j=  3,k=  2,DATAPACKING="POINT"'
    assert len(lines) == 3 + 24
    assert lines[3 + 5] == "   1.000000   1.000000   0.000000  0.500000000000000E+01"
