"""Mixed-precision path (CHAN_MIXED): float stage storage and fluxes, double
step state, RK accumulation, T/p recovery, forcing, wall BC and reductions.

Its results are not bit-parity results: the error against the FP64 oracle is
measured and bounded here, per step, as a relative L2 norm per variable
(||mixed - fp64|| / ||fp64|| over var(1:nP1,1:nP2,1:nP3,1:7)).
"""
import numpy as np
import pytest

from chan_cases import make_case
from compchan3dmpi_b200 import Channel, ChanError, RK3
from compchan3dmpi_b200 import wallbc as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
# relative L2 bound per variable over the first 200 steps.  v and w are the
# small perturbation components, whose own norms decay, so their relative
# error is also bounded against the streamwise velocity's norm.
MIXED_TOL = np.array([1e-4, 1e-4, 1e-3, 1e-3, 1e-4, 1e-4, 1e-4])
VEL_TOL = 1e-4


def rel_l2(a, b):
    return np.array([np.linalg.norm(a[m] - b[m]) / np.linalg.norm(b[m]) for m in range(a.shape[0])])


def test_mixed_error_against_fp64_oracle_200_steps():
    p, x3, jac, inv, var = make_case(nP=(32, 24, 33), mesh="tanh", beta=2.2, rk=RK3, Pr=0.72, istat=10, cfl=0.6)
    g = Channel(p.with_(mixed=True), x3, jac, inv)
    g.init_sol_v(var)
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    worst = np.zeros(7)
    for blk in range(20):
        g.step(10)
        o.step(10)
        gv, ov = g.download(), o.download()
        e = rel_l2(gv, ov)
        worst = np.maximum(worst, e)
        assert np.all(e <= MIXED_TOL), f"step {10 * (blk + 1)}: {e}"
        un = np.linalg.norm(ov[1])
        for m in (1, 2, 3):   # velocity errors against the streamwise velocity's norm
            assert np.linalg.norm(gv[m] - ov[m]) / un <= VEL_TOL, (10 * (blk + 1), m)
    assert worst.max() > 0.0          # the path really runs in reduced precision
    gt, g1, _, _ = g.stats()
    ot, o1, _, _ = o.stats()
    assert np.all(np.abs(gt - ot) <= 1e-4 * np.max(np.abs(ot)))
    for r in range(7):   # plane means against the row's scale; velocities against u's
        scale = np.max(np.abs(o1[1])) if r in (1, 2, 3) else np.max(np.abs(o1[r]))
        assert np.max(np.abs(g1[r] - o1[r])) <= 1e-4 * scale, r


def test_mixed_runs_whole_steps_only_and_restarts_exactly(tmp_path):
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), quantize=False, istat=3)
    pm = p.with_(mixed=True)
    a = Channel(pm, x3, jac, inv)
    a.init_sol_v(var)
    with pytest.raises(ChanError) as ei:
        a.stage(1)
    assert ei.value.code == -4
    a.step(8)
    ref = a.download()
    b = Channel(pm, x3, jac, inv)
    b.init_sol_v(var)
    b.step(4)
    b.checkpoint_write(tmp_path / "m.ckp")
    c = Channel(pm, x3, jac, inv)
    c.checkpoint_read(tmp_path / "m.ckp")
    c.step(4)
    assert np.array_equal(c.download(), ref)
    assert a.debug_canaries() == 0 and c.debug_canaries() == 0


@pytest.mark.parametrize("name", ["st4", "gst2", "s3", "rd1"])
def test_mixed_wall_variants_track_fp64(name):
    p, x3, jac, inv, var = make_case(nP=(24, 16, 21), mesh="tanh", beta=2.0, rk=RK3, Pr=0.72, istat=5,
                                     quantize=False)
    bottom, top = W.reference_variant(name, p)
    g = Channel(p.with_(mixed=True), x3, jac, inv)
    g.init_sol_v(var)
    g.set_wall_bc(0, bottom); g.set_wall_bc(1, top)
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    o.set_wall_bc(0, bottom); o.set_wall_bc(1, top)
    g.step(20)
    o.step(20)
    assert np.all(rel_l2(g.download(), o.download()) <= MIXED_TOL)


def test_mixed_check_long_run_profiles_small_grid():
    """mixed_check.compare on a small grid: the averaged profiles in wall units
    (Cf, u+, rms, <u'w'>) of the mixed path stay close to the FP64 path's."""
    from compchan3dmpi_b200 import mixed_check
    p, x3, jac, inv, var = make_case(nP=(32, 24, 33), mesh="tanh", beta=2.2, rk=RK3, Pr=0.72, istat=10, cfl=0.6)
    # this coarse grid stays stable for about 240 steps
    r = mixed_check.compare(p, x3, jac, inv, var, steps=200, avg_from=100, every=50)
    assert [s["step"] for s in r["series"]] == [50, 100, 150, 200]
    for s in r["series"]:
        assert np.all(np.array(s["rel_l2"]) <= MIXED_TOL), s
    pr = r["profiles"]
    assert pr["samples"] == 10
    assert pr["Cf"]["fp64"] > 0 and pr["Cf"]["rel_err"] <= 1e-4
    assert pr["uplus_rel_err"] <= 1e-4
    for v in ("rho", "u", "E", "T", "p"):
        assert pr["mean_rel_err"][v] <= 1e-4, v
    assert pr["rms_rel_err"]["u"] <= 1e-3
    assert pr["uw_rel_err"] <= 1e-3
    assert r["wall_s"]["fp64"] > 0 and r["wall_s"]["mixed"] > 0


def test_mixed_production_grid_against_fp64():
    """Mixed precision on the benchmark grid (256, 192, 193): 50 steps against
    the plain FP64 path from the same start, relative L2 per variable within
    the small-grid bounds; the time-averaged wall shear within 1e-5."""
    from compchan3dmpi_b200 import production_params, mesh_tanh, laminar_noise, cfl_dt
    nP = (256, 192, 193)
    x3, jac, inv = mesh_tanh(nP[2], 2.2)
    p = production_params(nP)
    var = laminar_noise(p, x3, seed=1234)
    p = p.with_(dt=cfl_dt(var, p, jac, 0.6))
    a = Channel(p.with_(mixed=True), x3, jac, inv)
    b = Channel(p, x3, jac, inv)
    for ch in (a, b):
        ch.init_sol_v(var)
        ch.time_avg_start()
        ch.step(50)
    e = rel_l2(a.download(), b.download())
    assert np.all(e <= MIXED_TOL), e
    ta, tb = a.time_average()["tau"], b.time_average()["tau"]
    assert np.all(np.abs(ta - tb) <= 1e-5 * np.max(np.abs(tb)))
    a.close()
    b.close()


def test_mixed_with_the_reference_rk2_scheme():
    """Mixed precision under the reference's two-stage RK (stage 1 double in,
    float out; stage 2 float in, double out) against the oracle over 100 steps
    of the reference grid's physics on a small grid."""
    from compchan3dmpi_b200 import RK2
    p, x3, jac, inv, var = make_case(nP=(32, 24, 33), mesh="cosine", rk=RK2, Pr=0.71, istat=10, cfl=0.5)
    g = Channel(p.with_(mixed=True), x3, jac, inv)
    g.init_sol_v(var)
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    for blk in range(4):
        g.step(25)
        o.step(25)
        e = rel_l2(g.download(), o.download())
        assert np.all(e <= MIXED_TOL), (25 * (blk + 1), e)
    assert e.max() > 0.0


def test_mixed_buoyancy_tracks_fp64():
    """The buoyancy term on the mixed path (computed in double from the float
    stage state) against the plain FP64 path with the same term."""
    from compchan3dmpi_b200.ensemble import stratified_start
    p, x3, jac, inv, _ = make_case(nP=(24, 16, 21), mesh="tanh", beta=2.2, rk=RK3, Pr=0.72, istat=5, quantize=False)
    p = p.with_(Tw=(0.9, 1.1))
    var = stratified_start(p, x3, 0.9, 1.1, seed=99)
    a = Channel(p.with_(mixed=True), x3, jac, inv)
    b = Channel(p, x3, jac, inv)
    for ch in (a, b):
        ch.set_buoyancy(0.5, 1.0)
        ch.init_sol_v(var)
        ch.step(40)
    assert np.all(rel_l2(a.download(), b.download()) <= MIXED_TOL)
