"""CPU tests of the host-side pieces: seeded IC, mesh options, deck formats."""
import math

import numpy as np
import pytest

from compchan3dmpi_b200 import (ChanParams, laminar_noise, mesh_cosine, mesh_tanh, cfl_dt, periodic_coords,
                                wall_coeffs)
from compchan3dmpi_b200.deck import (fmt_e22_15, parse_fortran_real, quantize_deck, write_param_dat,
                                     read_param_dat, write_3d_dat, read_3d_dat, DeckError)


def test_ic_is_seeded_periodic_and_consistent():
    p = ChanParams(nP=(18, 10, 13))
    x3, _, _ = mesh_cosine(13)
    a = laminar_noise(p, x3, seed=7)
    b = laminar_noise(p, x3, seed=7)
    c = laminar_noise(p, x3, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    # periodic duplicates (mainV1.8_serial.f90:162-170)
    assert np.array_equal(a[..., 0], a[..., -2]) and np.array_equal(a[..., -1], a[..., 1])
    assert np.array_equal(a[:, :, 0], a[:, :, -2]) and np.array_equal(a[:, :, -1], a[:, :, 1])
    # walls at rest, T = Tw
    assert np.all(a[1:4, 0] == 0) and np.all(a[1:4, -1] == 0) and np.all(a[5, 0] == 1.0)
    # equation of state and energy as main_v1.9.f90:605-606
    np.testing.assert_allclose(a[6], a[0] * a[5] / (1.4 * 1.5 ** 2), rtol=1e-15)
    ke = 0.5 * p.ggM * (a[1] ** 2 + a[2] ** 2 + a[3] ** 2)
    np.testing.assert_allclose(a[4] - ke, a[5], rtol=1e-14)
    # noise amplitude bounded by 10 % of the laminar profile
    ulam = 1.5 * (1 - (x3 - 1) ** 2)
    assert np.all(np.abs(a[2]) <= 0.1 * ulam[:, None, None] + 1e-15)


def test_tanh_mesh():
    x3, jac, inv = mesh_tanh(193, 2.2)
    assert x3[0] == 0.0 and x3[-1] == 2.0 and np.all(np.diff(x3) > 0)
    # analytic jacobian vs finite difference of the map
    dxi = 2.0 / 192
    fd = (x3[2:] - x3[:-2]) / (2 * dxi)
    np.testing.assert_allclose(fd, jac[1:-1], rtol=2e-3)
    np.testing.assert_allclose(inv, 1.0 / jac)
    assert abs(np.sum(0.5 * (jac[1:] + jac[:-1])) * dxi - 2.0) < 1e-3


def test_cfl_dt_scales_linearly():
    p = ChanParams(nP=(16, 12, 17))
    x3, jac, _ = mesh_cosine(17)
    var = laminar_noise(p, x3)
    d5 = cfl_dt(var, p, jac, 0.5)
    d1 = cfl_dt(var, p, jac, 1.0)
    assert d5 > 0 and abs(d1 / d5 - 2.0) < 1e-12


def test_e22_15_format():
    assert fmt_e22_15(0.0) == " 0.000000000000000E+00"
    assert fmt_e22_15(1.0) == " 0.100000000000000E+01"
    assert fmt_e22_15(-0.00123456789012345678) == "-0.123456789012346E-02"
    assert len(fmt_e22_15(math.pi)) == 22
    assert parse_fortran_real("0.314159265358979E+01") == 3.14159265358979
    assert parse_fortran_real("0.1+100") == 1e99
    q = quantize_deck(np.array([math.pi, -1e-7 / 3]))
    assert q[0] == 3.14159265358979 and q[1] == float("-0.333333333333333E-07")


def test_param_dat_roundtrip(tmp_path):
    p = ChanParams(nP=(64, 48, 65), Re=3000.0, Mac=1.5, dt=1e-4, istat=10, Pe=(2.0, 2.0, 0.2))
    f = tmp_path / "param.dat"
    write_param_dat(f, p, descp="case4", topo=(2, 2, 2), inputPath="../input/3D.dat")
    text = f.read_text().splitlines()
    # values start at column 49 (48X in comdata.f90:37-55)
    assert text[10][48:52] == "3000"[:4] or text[10][48:52].strip() == "3000."
    q, ex = read_param_dat(f, nP=(64, 48, 65))
    assert (q.Re, q.Mac, q.dt, q.istat, q.Pe) == (3000.0, 1.5, 1e-4, 10, (2.0, 2.0, 0.2))
    assert ex["topo"] == (2, 2, 2) and ex["inputPath"] == "../input/3D.dat" and ex["descp"] == "case4"


def test_param_dat_small_dt_uses_exponent(tmp_path):
    p = ChanParams(dt=3.7e-5)
    f = tmp_path / "param.dat"
    write_param_dat(f, p)
    q, _ = read_param_dat(f)
    assert abs(q.dt - 3.7e-5) < 1e-10


def test_3d_dat_roundtrip_and_errors(tmp_path):
    p = ChanParams(nP=(6, 6, 7))
    x3, _, _ = mesh_cosine(7)
    v = quantize_deck(laminar_noise(p, x3))
    f = tmp_path / "3D.dat"
    write_3d_dat(f, v, periodic_coords(6, p.Lx), periodic_coords(6, p.Ly), x3, 1.25, 42)
    back, t, n, x1, x2, x3b = read_3d_dat(f, p.nP)
    assert np.array_equal(back, v) and t == 1.25 and n == 42
    assert np.allclose(x3b, x3, atol=1e-6)
    # a truncated file is reported with the record's indices, like the reference
    lines = f.read_text().splitlines()
    (tmp_path / "bad.dat").write_text("\n".join(lines[:40]) + "\n")
    with pytest.raises(DeckError, match="Error in reading combined input file"):
        read_3d_dat(tmp_path / "bad.dat", p.nP)
    # a corrupt number too
    bad = lines[:]
    bad[10] = bad[10][:40] + "x" + bad[10][41:]
    (tmp_path / "bad2.dat").write_text("\n".join(bad) + "\n")
    with pytest.raises(DeckError):
        read_3d_dat(tmp_path / "bad2.dat", p.nP)


def test_wall_coeffs_sum_to_zero():
    x3, _, _ = mesh_cosine(65)
    c = wall_coeffs(x3)
    assert abs(c["f1d2c0"] + c["f1d2c1"] + c["f1d2c2"]) < 1e-9 * abs(c["f1d2c0"])
    assert abs(c["b1d2c0"] + c["b1d2c1"] + c["b1d2c2"]) < 1e-9 * abs(c["b1d2c0"])


def test_wall_units_laminar_known_answer():
    """Poiseuille u = 1.5(1-(z-1)^2), rho = T = 1: tau_w = mu*du/dz/Re = 3/Re,
    U_b = 1, so Cf = 6/Re and u_tau = sqrt(3/Re)."""
    from compchan3dmpi_b200.stats import wall_units
    x3, _, _ = mesh_cosine(401)
    Re = 3000.0
    mean = np.zeros((7, x3.size))
    mean[0] = 1.0
    mean[1] = 1.5 * (1 - (x3 - 1) ** 2)
    w = wall_units(mean, np.array([3.0 / Re, -3.0 / Re]), x3, Re)
    assert abs(w["Cf"] - 6.0 / Re) < 1e-4 * (6.0 / Re)   # trapezoidal U_b on 401 points
    assert abs(w["u_tau"] - math.sqrt(3.0 / Re)) < 1e-15
    assert abs(w["Re_tau"] - math.sqrt(3.0 * Re)) < 1e-9
    assert w["yplus"][0] == 0.0 and w["uplus"][0] == 0.0


def test_time_average_formulas_and_series_roundtrip(tmp_path):
    """avg_v1.7.f90:239-274 on synthetic snapshots; series files in the reference's F15.7 format."""
    from compchan3dmpi_b200.stats import average_snapshots, append_series, read_series, write_profiles
    rng = np.random.default_rng(3)
    n3 = 6
    snaps = []
    for s in range(4):
        s1 = rng.uniform(0.5, 1.5, (7, n3)); s2 = s1 ** 2 + rng.uniform(0, 0.1, (7, n3))
        c = rng.uniform(0, 1, (9, n3)); tau = rng.uniform(-1e-3, 1e-3, 2)
        snaps.append((s1, s2, c, tau))
        append_series(tmp_path, 0.1 * (s + 1), tau, s1, s2, c)
    mean, rms, covar, tau = average_snapshots(snaps)
    m1 = sum(s[0] for s in snaps) / 4
    assert np.allclose(mean, m1)
    assert np.allclose(rms, np.sqrt(sum(s[1] for s in snaps) / 4 - m1 ** 2))
    assert np.allclose(covar[2], sum(s[2][2] for s in snaps) / 4 - m1[1] * m1[2])
    t, v = read_series(tmp_path / "moment1st.dat", 7, n3)
    assert np.allclose(t, [0.1, 0.2, 0.3, 0.4]) and np.allclose(v[0], snaps[0][0], atol=5e-8)
    write_profiles(tmp_path, np.linspace(0, 2, n3), mean, rms, covar)
    assert len((tmp_path / "mean.dat").read_text().splitlines()) == n3


def test_native_deck_matches_python_byte_for_byte(tmp_path):
    from compchan3dmpi_b200.deck import write_3d_dat_native, read_3d_dat_native
    p = ChanParams(nP=(9, 6, 7))
    x3, _, _ = mesh_cosine(7)
    v = quantize_deck(laminar_noise(p, x3))
    v[4, 3, 2, 1] = -1.2345678901234567e-120   # three-digit exponent form
    v[2, 0, 0, 0] = 0.0
    x1, x2 = periodic_coords(9, p.Lx), periodic_coords(6, p.Ly)
    write_3d_dat(tmp_path / "py.dat", v, x1, x2, x3, 0.375, 17)
    write_3d_dat_native(tmp_path / "c.dat", v, x1, x2, x3, 0.375, 17, threads=3)
    assert (tmp_path / "py.dat").read_bytes() == (tmp_path / "c.dat").read_bytes()
    back, t, n, bx1, bx2, bx3 = read_3d_dat_native(tmp_path / "c.dat", p.nP, threads=2)
    pyb, pt, pn, *_ = read_3d_dat(tmp_path / "c.dat", p.nP)
    assert np.array_equal(back, pyb) and t == pt == 0.375 and n == pn == 17
    assert np.allclose(bx3, x3, atol=1e-6) and np.allclose(bx1, x1, atol=1e-6)


def test_native_deck_reports_bad_records(tmp_path):
    from compchan3dmpi_b200.deck import write_3d_dat_native, read_3d_dat_native
    p = ChanParams(nP=(6, 6, 7))
    x3, _, _ = mesh_cosine(7)
    v = laminar_noise(p, x3)
    f = tmp_path / "3D.dat"
    write_3d_dat_native(f, v, periodic_coords(6, p.Lx), periodic_coords(6, p.Ly), x3)
    lines = f.read_text().splitlines()
    (tmp_path / "short.dat").write_text("\n".join(lines[:50]) + "\n")
    with pytest.raises(DeckError, match="Error in reading combined input file at"):
        read_3d_dat_native(tmp_path / "short.dat", p.nP)
    bad = lines[:]
    bad[12] = bad[12][:60] + "#" + bad[12][61:]
    (tmp_path / "bad.dat").write_text("\n".join(bad) + "\n")
    with pytest.raises(DeckError, match="Error in reading combined input file at 1 2 1"):   # line 12 = i1 j2 k1
        read_3d_dat_native(tmp_path / "bad.dat", p.nP)
    with pytest.raises(DeckError, match="cannot open"):
        read_3d_dat_native(tmp_path / "missing.dat", p.nP)


def test_driver_event_cadence_and_debug_format(tmp_path):
    from compchan3dmpi_b200.run import _next_event, write_debug_dump
    assert _next_event(0, 50, 7) == 7
    assert _next_event(7, 50, 7) == 10
    assert _next_event(995, 5000, 0) == 1000
    assert _next_event(48, 50, 10) == 50
    var = np.zeros((7, 2, 2, 2)); var[0] = 1.5; var[5] = -2.5e-3
    write_debug_dump(tmp_path / "d.dat", var, [0.0, 1.0], [0.0, 0.5], [0.0, 2.0], 0.25, 7)
    lines = (tmp_path / "d.dat").read_text().splitlines()
    assert lines[0] == 'TITLE ="        0.2500000000        7"'
    assert lines[5] == "  0.0000  0.0000  0.0000  0.15000E+01  0.00000E+00  0.00000E+00  0.00000E+00" \
                       "  0.00000E+00 -0.25000E-02  0.00000E+00"


def test_mixed_check_rejects_bad_windows_before_any_device_work():
    from compchan3dmpi_b200 import mixed_check, production_params
    p = production_params((20, 14, 19), istat=10)
    for steps, avg_from, every in ((1000, 500, 300), (1000, 1000, 100), (1000, 200, 15), (950, 100, 100)):
        with pytest.raises(ValueError):
            mixed_check.compare(p, None, None, None, None, steps, avg_from, every)


def test_sweep_cases_cover_the_parameter_grid_and_are_seeded():
    from compchan3dmpi_b200.ensemble import sweep_cases, sweep_grids, MACH, REYNOLDS, RICHARDSON, DELTA_T
    g = sweep_grids(16)
    assert g[0] == (64, 64, 65)
    assert max(n[0] for n in g) == 160 and max(n[1] for n in g) == 128 and max(n[2] for n in g) == 129
    assert len(set(g)) == 16 and all(n[2] % 2 == 1 for n in g)
    a = sweep_cases(16, grids=[(24, 16, 17)] * 16)
    b = sweep_cases(16, grids=[(24, 16, 17)] * 16)
    combos = {(c.params.Mac, c.params.Re, c.Ri, c.dT) for c in a}
    assert len(combos) == 16          # drawn without repetition
    for c in a:
        assert c.params.Mac in MACH and c.params.Re in REYNOLDS and c.Ri in RICHARDSON and c.dT in DELTA_T
        assert c.params.Tw == (1.0 - 0.5 * c.dT, 1.0 + 0.5 * c.dT)
        assert c.params.mixed and c.params.dt > 0
    for x, y in zip(a, b):
        assert np.array_equal(x.var, y.var) and x.params == y.params


def test_stratified_start_is_at_uniform_pressure():
    from compchan3dmpi_b200.ensemble import stratified_start
    p = ChanParams(nP=(12, 10, 13), Tw=(0.9, 1.1))
    x3, jac, inv = mesh_tanh(13, 2.2)
    v = stratified_start(p, x3, 0.9, 1.1, seed=5)
    assert np.allclose(v[5][0], 0.9) and np.allclose(v[5][-1], 1.1)
    assert np.allclose(v[6], 1.0 / (p.gama * p.Mac ** 2))
    assert np.allclose(v[0] * v[5], 1.0)
    assert np.allclose(v[4], v[5] + 0.5 * p.ggM * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2))


def test_closure_coarsening_and_smooth_start():
    """The coarse start of the closure experiment: periodic linear
    interpolation is exact on the coarse grid's own points when they are a
    subset of the source's, every third wall-normal plane of a tanh grid is the
    coarse tanh grid, walls come out at rest at their temperature, and E and p
    follow from the primitives."""
    from compchan3dmpi_b200.closure import coarsen, smooth_start, _interp_periodic
    n = 2 + 48
    src = np.sin(2 * np.pi * np.arange(-1, n - 1) / (n - 2))[None, :]
    dst = _interp_periodic(src, n, 2 + 12, axis=-1)[0]
    assert np.allclose(dst[1:-1], np.sin(2 * np.pi * np.arange(12) / 12), atol=1e-12)
    assert dst[0] == dst[-2] and dst[-1] == dst[1]
    pd = ChanParams(nP=(50, 26, 25), Tw=(0.9, 1.1))
    pc = ChanParams(nP=(14, 8, 9), Tw=(0.9, 1.1))
    x3d, _, _ = mesh_tanh(25, 2.2)
    x3c, _, _ = mesh_tanh(9, 2.2)
    assert np.allclose(x3d[::3], x3c)
    v = smooth_start(pd, x3d)
    assert np.all(np.isfinite(v)) and np.abs(v[1]).max() > 1.0
    c = coarsen(v, pd, pc, 3)
    assert c.shape == (7, 9, 8, 14)
    assert np.all(c[1:4, 0] == 0) and np.all(c[1:4, -1] == 0)
    assert np.all(c[5, 0] == 0.9) and np.all(c[5, -1] == 1.1)
    assert np.allclose(c[4], c[5] + 0.5 * pc.ggM * (c[1] ** 2 + c[2] ** 2 + c[3] ** 2))
    assert np.allclose(c[6], c[0] * c[5] / (pc.gama * pc.Mac ** 2))
    # periodic duplicates of the coarse field
    assert np.array_equal(c[..., 0], c[..., -2]) and np.array_equal(c[..., -1], c[..., 1])


def test_closure_deficit_targets_and_magnitude_knob():
    """The a-posteriori targets: each sample's tau_uw gets the deficit of the
    coarse plane it sits on (samples in snapshots, planes in order); the
    magnitude knob scales only the output half of the normalisation; the
    stationarity measure sees a drift."""
    from compchan3dmpi_b200.closure import add_shear_deficit, scaled_norm, stationarity

    class Fake:
        def __init__(self, X=None, T=None):
            self.X = [] if X is None else [X]
            self.T = [] if T is None else [T]

        @property
        def count(self):
            return sum(len(x) for x in self.X)

        def data(self, first, n):
            X, T = np.concatenate(self.X), np.concatenate(self.T)
            return X[first:first + n].copy(), T[first:first + n].copy()

        def add_data(self, X, T):
            self.X.append(X)
            self.T.append(T)

    per_plane, planes, snaps = 5, 3, 2
    n = per_plane * planes * snaps
    X = np.arange(n * 13, dtype=np.float32).reshape(n, 13)
    T = np.zeros((n, 9), np.float32)
    deficit = np.array([99.0, 1.0, 2.0, 3.0, 99.0])   # coarse planes 0..4; interior 1..3
    src, dst = Fake(X, T), Fake()
    add_shear_deficit(src, dst, deficit, per_plane * planes, per_plane, chunk=7)
    X2, T2 = dst.data(0, n)
    assert np.array_equal(X2, X)
    want = np.tile(np.repeat([1.0, 2.0, 3.0], per_plane), snaps)
    assert np.array_equal(T2[:, 4], want.astype(np.float32))
    assert np.all(np.delete(T2, 4, axis=1) == 0)
    norm = np.arange(44, dtype=np.float32)
    s = scaled_norm(norm, 2.0)
    assert np.array_equal(s[:26], norm[:26]) and np.array_equal(s[26:], 2 * norm[26:])
    flat = stationarity([(t, 1.0) for t in range(10)])
    rising = stationarity([(t, 1.0 + 0.1 * t) for t in range(10)])
    assert abs(flat["drift"]) < 1e-12 and rising["drift"] > 0.3 and rising["halves"] > 0.2


def test_closure_runs_over_several_seeds_combine():
    """Coarse runs from several seeds: statistics averaged run by run, profiles
    point by point; a run that fell back or blew up leaves no statistics and
    its report is the one kept."""
    from compchan3dmpi_b200.closure import mean_stats, seed_runs
    ok = {"fallback_step": None, "reason": None, "plain_failed": None}
    a = {"steps": 10, "wall_s": 1.0, "report": ok, "stats": {"Cf": 1.0, "uw": [0.0, 2.0]}}
    b = {"steps": 10, "wall_s": 3.0, "report": ok, "stats": {"Cf": 2.0, "uw": [1.0, 4.0]}}
    m = mean_stats([a["stats"], b["stats"]])
    assert m == {"Cf": 1.5, "uw": [0.5, 3.0]}
    r = seed_runs([a, b])
    assert r["stats"] == m and r["wall_s"] == 2.0 and r["report"] == ok and len(r["per_seed"]) == 2
    fell = {"steps": 10, "wall_s": 2.0, "stats": {"Cf": 9.0, "uw": [9.0, 9.0]},
            "report": {"fallback_step": 400, "reason": "closure output beyond its limit", "plain_failed": None}}
    r = seed_runs([a, fell])
    assert r["stats"] is None and r["report"]["fallback_step"] == 400
