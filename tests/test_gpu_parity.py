"""Parity of the sm_100a library (through its C ABI) with the oracle.

Tolerance: the plain FP64 path must match the oracle to <= 1e-12 relative
per step.  The metric is the per-variable normwise error max|d| / max|ref|
over var(1:nP1,1:nP2,1:nP3,1:7).  The two sides differ only by rounding: the
GPU forms stencils as weighted sums with FMA, uses reciprocal
multiplication, and derives the first stage's primitives from the
conservative state.
"""
import numpy as np
import pytest

from chan_cases import CASES, make_case, rel_err, worst
from compchan3dmpi_b200 import Channel, BlowUpError, RK2, RK3, FORCE_NONE
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _pair(case):
    p, x3, jac, inv, var = case
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    return g, o


def _assert_close(gv, ov, tol=TOL, what=""):
    e = rel_err(gv, ov)
    assert e.max() <= tol, f"{what}: per-variable error {e} worst at {worst(gv, ov)}"
    return e


def test_upload_download_roundtrip():
    case = make_case(**CASES["ref_rk2_cosine"])
    g, o = _pair(case)
    # download right after upload returns the reference's var after initSolV+share2P.
    # rho,u,v,w,E come back to the last bit of the deck; T and p are re-derived
    # from the conservative state, and the deck's 15-digit E and T are not
    # exactly consistent (E ~ 2.7 carries ~5e-15 absolute rounding), hence 1e-13.
    e = rel_err(g.download(), o.download())
    assert e[:5].max() <= 2e-16, e
    assert e[5:].max() <= 1e-13, e


@pytest.mark.parametrize("name", list(CASES))
def test_single_stage(name):
    case = make_case(**CASES[name])
    g, o = _pair(case)
    g.stage(1)
    o.stage(1)
    _assert_close(g.download(), o.download(), what=f"{name} stage 1")


@pytest.mark.parametrize("name", list(CASES))
def test_steps_per_step(name):
    case = make_case(**CASES[name])
    g, o = _pair(case)
    for s in range(1, 7):
        g.step(1)
        o.step(1)
        _assert_close(g.download(), o.download(), what=f"{name} step {s}")
    assert g.nstep == o.nstep == 6
    assert g.time == o.time


def test_stats_and_forcing():
    """istat=2: tau_w and plane moments feed the forcing from step 3 on."""
    case = make_case(**CASES["ref_rk2_cosine"])
    g, o = _pair(case)
    g.step(4)
    o.step(4)
    gt, g1, g2, gc = g.stats()
    ot, o1, o2, oc = o.stats()
    assert np.all(np.abs(gt - ot) <= 1e-12 * np.max(np.abs(ot))), (gt, ot)
    for a, b in ((g1, o1), (g2, o2), (gc, oc)):
        for r in range(a.shape[0]):
            den = max(np.max(np.abs(b[r])), 1e-300)
            assert np.max(np.abs(a[r] - b[r])) <= 1e-12 * den
    assert abs(ot[0] - ot[1]) > 0  # the forcing is active in this case
    _assert_close(g.download(), o.download(), what="after forcing")


def test_reference_grid_64x48x65_100_steps():
    """Reference physics on the 64 x 48 x 65 grid (x, spanwise, wall-normal), 100 RK2 steps."""
    case = make_case(nP=(64, 48, 65), mesh="cosine", rk=RK2, Pr=0.71, istat=10, quantize=False)
    g, o = _pair(case)
    for blk in range(4):
        g.step(25)
        o.step(25)
        _assert_close(g.download(), o.download(), what=f"64x48x65 step {25 * (blk + 1)}")


def test_grid_64x48x65_tanh_rk3_cfl05_100_steps():
    """The 64 x 65 x 48 case as specified for the CPU-runnable comparison: tanh
    wall stretching beta = 2, SSP-RK3 at CFL 0.5, Pr 0.72, seeded +-10% start,
    100 steps, compared with the oracle every 25 steps."""
    case = make_case(nP=(64, 48, 65), mesh="tanh", beta=2.0, rk=RK3, Pr=0.72, istat=10, cfl=0.5, quantize=False)
    g, o = _pair(case)
    for blk in range(4):
        g.step(25)
        o.step(25)
        _assert_close(g.download(), o.download(), what=f"64x48x65 tanh RK3 step {25 * (blk + 1)}")
    gt, g1, _, _ = g.stats()
    ot, o1, _, _ = o.stats()
    assert np.all(np.abs(gt - ot) <= 1e-12 * np.max(np.abs(ot)))


def test_tau_and_avg_explicit_calls():
    case = make_case(**CASES["rk3_tanh"])
    g, o = _pair(case)
    g.step(1); o.step(1)
    g.calc_tau_wall(); o.tau_wall()
    g.avg_spatial(); o.avg_spatial()
    gt, g1, _, _ = g.stats()
    ot, o1, _, _ = o.stats()
    np.testing.assert_allclose(gt, ot, rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(g1, o1, rtol=1e-12, atol=1e-15)


def test_set_forcing_matches():
    case = make_case(**CASES["ref_rk2_cosine"])
    p = case[0]
    g, o = _pair(case)
    rb = np.linspace(0.99, 1.01, p.nP[2])
    g.set_forcing(2e-3, -1e-3, rb)
    o.set_forcing(2e-3, -1e-3, rb)
    g.step(2); o.step(2)
    _assert_close(g.download(), o.download(), what="set_forcing")


def test_no_forcing_switch():
    case = make_case(nP=(20, 14, 19), forcing=FORCE_NONE, istat=1)
    g, o = _pair(case)
    g.step(3); o.step(3)
    _assert_close(g.download(), o.download(), what="no forcing")


def test_blowup_reported_like_reference():
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), quantize=False)
    var = var.copy()
    var[0, 6, 5, 7] = -1.0
    g, o = _pair((p, x3, jac, inv, var))
    with pytest.raises(BlowUpError) as ei:
        g.step(5)
    assert o.step(5) == 1
    assert ei.value.nstep == 1 == o.nstep
    i, j, k = ei.value.ijk
    ov = o.download()
    assert ov[0, k - 1, j - 1, i - 1] < 0 or ov[5, k - 1, j - 1, i - 1] < 0
    # the state is frozen at the step that blew up: further steps do nothing
    before = g.download()
    with pytest.raises(BlowUpError):
        g.step(1)
    assert np.array_equal(g.download(), before)


def test_nonfinite_status():
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), quantize=False)
    var = var.copy()
    var[1, 8, 6, 9] = np.nan
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    assert g.step(1) == 2   # CHAN_NONFINITE


def test_deck_file_roundtrip(tmp_path):
    from compchan3dmpi_b200.deck import write_3d_dat
    from compchan3dmpi_b200 import periodic_coords
    p, x3, jac, inv, var = make_case(nP=(12, 8, 9))
    path = tmp_path / "3D.dat"
    write_3d_dat(path, var, periodic_coords(12, p.Lx), periodic_coords(8, p.Ly), x3, 0.0, 0)
    g = Channel(p, x3, jac, inv)
    v2 = g.read_input_file(path)
    assert np.array_equal(v2, var)
    g.step(2)
    g.write_soln(tmp_path / "out.dat")
    from compchan3dmpi_b200.deck import read_3d_dat
    back, t, n, *_ = read_3d_dat(tmp_path / "out.dat", p.nP)
    assert n == 2 and abs(t - 2 * p.dt) < 1e-10   # time is written as F20.10
    np.testing.assert_allclose(back, g.download(), rtol=1e-14, atol=1e-300)


def test_errors_are_codes():
    from compchan3dmpi_b200 import ChanError
    p, x3, jac, inv, var = make_case(nP=(12, 8, 9))
    g = Channel(p, x3, jac, inv)
    with pytest.raises(ChanError) as ei:
        g.stage(1)   # before upload
    assert ei.value.code == -4
    with pytest.raises(ChanError):
        Channel(p.with_(nP=(4, 8, 9)), x3[:9], jac[:9], inv[:9])


def test_time_averaged_statistics_match_oracle():
    """Device-side time averaging (avg_v1.7.f90:239-274) against averages of the
    oracle's plane statistics captured at every statistics step."""
    from compchan3dmpi_b200.stats import average_snapshots, wall_units
    p, x3, jac, inv, var = make_case(nP=(24, 16, 21), quantize=False, istat=2)
    g, o = _pair((p, x3, jac, inv, var))
    g.time_avg_start()
    snaps = []
    for s in range(1, 9):
        g.step(1)
        o.step(1)
        if s % p.istat == 0:
            snaps.append(tuple(np.array(a) for a in (o.stats()[1], o.stats()[2], o.stats()[3], o.stats()[0])))
    ta = g.time_average()
    assert ta["samples"] == len(snaps) == 4
    mean, rms, covar, tau = average_snapshots(snaps)
    for r in range(mean.shape[0]):
        assert np.max(np.abs(ta["mean"][r] - mean[r])) <= 1e-12 * max(np.max(np.abs(mean[r])), 1e-300)
    # covariances are <ab> - <a><b>: differences of O(1) terms (rho, T, p ~ 1)
    # that cancel to ~1e-4, so the bound is 1e-12 of the row plus 1e-14 absolute
    for r in range(covar.shape[0]):
        assert np.max(np.abs(ta["covar"][r] - covar[r])) <= 1e-12 * np.max(np.abs(covar[r])) + 1e-14
    np.testing.assert_allclose(ta["rms"], rms, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(ta["tau"], tau, rtol=1e-12, atol=1e-20)
    w = wall_units(ta["mean"], ta["tau"], x3, p.Re)
    assert w["Cf"] > 0 and w["u_tau"] > 0


def test_checkpoint_restart_is_bit_exact(tmp_path):
    """8 steps straight == 4 steps, checkpoint, new context, restore, 4 steps."""
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), quantize=False, istat=3)
    a = Channel(p, x3, jac, inv)
    a.init_sol_v(var)
    a.time_avg_start()
    a.step(8)
    ref = a.download()
    ref_stats = a.stats()
    ref_avg = a.time_average()
    b = Channel(p, x3, jac, inv)
    b.init_sol_v(var)
    b.time_avg_start()
    b.step(4)
    b.checkpoint_write(tmp_path / "ck.bin")
    c = Channel(p, x3, jac, inv)
    c.checkpoint_read(tmp_path / "ck.bin")
    assert c.nstep == 4
    c.step(4)
    assert np.array_equal(c.download(), ref)
    for x, y in zip(c.stats(), ref_stats):
        assert np.array_equal(x, y)
    assert c.time_average()["samples"] == ref_avg["samples"]
    assert np.array_equal(c.time_average()["mean"], ref_avg["mean"])
    assert c.nstep == 8 and c.time == a.time


def test_checkpoint_faults_are_codes(tmp_path):
    """Truncated, foreign and mismatched checkpoint files are reported as codes and
    leave the context as it was (host-side fault injection)."""
    from compchan3dmpi_b200 import ChanError
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), quantize=False, istat=3)
    a = Channel(p, x3, jac, inv)
    a.init_sol_v(var)
    a.step(2)
    good = tmp_path / "good.ckp"
    a.checkpoint_write(good)
    blob = good.read_bytes()
    (tmp_path / "trunc.ckp").write_bytes(blob[: len(blob) // 2])
    (tmp_path / "foreign.ckp").write_bytes(b"NOTACKPT" + blob[8:])
    before = a.download()
    for name, code in (("trunc.ckp", -5), ("foreign.ckp", -5), ("missing.ckp", -5)):
        with pytest.raises(ChanError) as ei:
            a.checkpoint_read(tmp_path / name)
        assert ei.value.code == code, (name, ei.value)
        assert np.array_equal(a.download(), before)
    q2, x32, jac2, inv2, var2 = make_case(nP=(22, 14, 19), quantize=False)
    b = Channel(q2, x32, jac2, inv2)
    b.init_sol_v(var2)
    with pytest.raises(ChanError) as ei:
        b.checkpoint_read(good)
    assert ei.value.code == -1
    # same grid, other physics or method: refused, naming the field
    for change, field in ((dict(dt=p.dt * 0.5), "dt"), (dict(Re=p.Re + 1.0), "Re"),
                          (dict(rk_scheme=3 if p.rk_scheme == 2 else 2), "rk_scheme")):
        d = Channel(p.with_(**change), x3, jac, inv)
        with pytest.raises(ChanError) as ei:
            d.checkpoint_read(good)
        assert ei.value.code == -1 and field in str(ei.value), (change, str(ei.value))
        d.close()
    a.step(1)   # still usable
    assert a.nstep == 3



@pytest.mark.parametrize("Pe", [(1e300, 1e300, 1e300), (0.0, 0.0, 0.0)], ids=["central", "quick"])
def test_one_scheme_everywhere(Pe):
    """Pe thresholds never / always exceeded: the central and the QUICK branch alone."""
    case = make_case(nP=(20, 14, 19), Pe=Pe)
    g, o = _pair(case)
    for s in range(1, 4):
        g.step(1)
        o.step(1)
        _assert_close(g.download(), o.download(), what=f"Pe={Pe} step {s}")


@pytest.mark.parametrize("Pe", [(1e300, 1e300, 1e300), (0.0, 0.0, 0.0)], ids=["central", "quick"])
def test_plane_mass_conserved_on_gpu(Pe):
    """w = 0: each interior plane's mass over its periodic points is kept by a stage
    when one inviscid scheme is used everywhere (telescoping face fluxes)."""
    from chan_cases import conservation_case, plane_mass
    p, x3, jac, inv, var = conservation_case(Pe=Pe)
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    m0 = plane_mass(var)
    g.stage(1)
    m1 = plane_mass(g.download())
    rel = np.abs(m1[1:-1] - m0[1:-1]) / m0[1:-1]
    assert rel.max() <= 1e-13, rel.max()


@pytest.mark.parametrize("name", list(CASES))
def test_no_write_outside_buffers(name):
    """Guard zones around every state buffer stay intact through stages, steps,
    statistics, diagnostics, wall-BC plug-ins, downloads and checkpoints."""
    from compchan3dmpi_b200 import wallbc as W
    p, x3, jac, inv, var = make_case(**CASES[name])
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    assert g.debug_canaries() == 0
    g.diag_enable((3, 5, 70), every=2)
    g.time_avg_start()
    g.stage(1)
    g.step(3)
    g.set_wall_bc(0, W.reference_variant("gst3", p)[0])
    g.set_wall_bc(1, W.reference_variant("rd1", p)[0])
    g.step(4)
    g.calc_tau_wall(); g.avg_spatial(); g.stats(); g.diag_read(); g.time_average()
    g.fluctuation_q(np.ones((7, p.nP[2])))
    g.download()
    assert g.debug_canaries() == 0


def test_production_grid_matches_oracle():
    """The benchmark workload itself: nP = (256, 192, 193), tanh beta 2.2,
    SSP-RK3 at CFL 0.6, statistics every step; two steps on the GPU against
    the oracle on the full grid (about a second of host work)."""
    from compchan3dmpi_b200 import production_params, mesh_tanh, laminar_noise, cfl_dt
    nP = (256, 192, 193)
    x3, jac, inv = mesh_tanh(nP[2], 2.2)
    p = production_params(nP, istat=1)
    var = laminar_noise(p, x3, seed=1234)
    p = p.with_(dt=cfl_dt(var, p, jac, 0.6))
    g, o = _pair((p, x3, jac, inv, var))
    for s in (1, 2):
        g.step(1)
        o.step(1)
        gv, ov = g.download(), o.download()
        _assert_close(gv, ov, what=f"production grid step {s}")
        del gv, ov
    gt, g1, _, _ = g.stats()
    ot, o1, _, _ = o.stats()
    assert np.all(np.abs(gt - ot) <= 1e-12 * np.max(np.abs(ot)))
    for r in range(7):
        assert np.max(np.abs(g1[r] - o1[r])) <= 1e-12 * max(np.max(np.abs(o1[r])), 1e-300)
    g.close()
    o.close()
