"""Buoyancy term, stage-kernel launch shapes, ensembles and the launch-shape
autotuner, through the C ABI.

- The buoyancy term (chan_set_buoyancy) matches the oracle to the plain FP64
  path's 1e-12 per step.
- Launch shapes change no result bits: every tile shape and k-chunk count
  gives the same state as the default.
- An ensemble's members end bit for bit where the same contexts stepped
  alone end, across graph replays, remainder steps, statistics steps, time
  averaging and a setting changed between calls (which re-captures the graph).
- The autotuner leaves every member's state, counters and status as they
  were.
"""
import numpy as np
import pytest

from chan_cases import make_case, rel_err, worst
from compchan3dmpi_b200 import Channel, ChanError, RK3
from compchan3dmpi_b200 import _lib
from compchan3dmpi_b200 import wallbc as W
from compchan3dmpi_b200.ensemble import Ensemble, open_case, stratified_start, sweep_cases
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _strat_case(nP=(20, 14, 19), Tw=(0.9, 1.1), **kw):
    p, x3, jac, inv, var = make_case(nP=nP, mesh="tanh", beta=2.2, rk=RK3, Pr=0.72, istat=3, quantize=False, **kw)
    p = p.with_(Tw=Tw)
    var = stratified_start(p, x3, Tw[0], Tw[1], seed=99)
    return p, x3, jac, inv, var


def test_buoyancy_matches_oracle_per_step():
    p, x3, jac, inv, var = _strat_case()
    g = Channel(p, x3, jac, inv)
    g.set_buoyancy(0.5, 1.0)
    g.init_sol_v(var)
    o = O.Oracle(p, x3, jac, inv)
    o.set_buoyancy(0.5, 1.0)
    o.upload(var)
    for s in range(1, 9):
        g.step(1)
        o.step(1)
        gv, ov = g.download(), o.download()
        e = rel_err(gv, ov)
        assert e.max() <= TOL, f"step {s}: {e} worst at {worst(gv, ov)}"
    # and the term is really on: the run without it differs
    h = Channel(p, x3, jac, inv)
    h.init_sol_v(var)
    h.step(8)
    assert rel_err(h.download(), gv)[3] > 1e-8


@pytest.mark.parametrize("mixed", [False, True])
def test_launch_shapes_change_no_bits(mixed):
    p, x3, jac, inv, var = _strat_case(nP=(40, 20, 33))
    p = p.with_(mixed=mixed)
    ref = None
    shapes = [(0, 0), (0, 1), (0, 5), (0, 31), (1, 0), (1, 1), (1, 7), (2, 0), (2, 3), (3, 0), (3, 4)]
    for tile, nch in shapes:
        g = Channel(p, x3, jac, inv)
        g.set_buoyancy(0.1, 1.0)
        g.set_launch(tile, nch)
        t, n, k = g.launch()
        assert t == tile and (nch == 0 or n == -(-31 // -(-31 // nch)))
        assert n * k >= 31 and (n - 1) * k < 31
        g.init_sol_v(var)
        g.step(7)
        out = g.download()
        stats = g.stats()
        if ref is None:
            ref = (out, stats)
        else:
            assert np.array_equal(out, ref[0]), (tile, nch)
            for a, b in zip(stats, ref[1]):
                assert np.array_equal(a, b), (tile, nch)
        g.close()


def test_launch_shape_rejects_bad_values():
    p, x3, jac, inv, var = _strat_case()
    g = Channel(p, x3, jac, inv)
    for tile, nch in ((4, 0), (-1, 0), (0, -1), (0, 18)):
        with pytest.raises(ChanError):
            g.set_launch(tile, nch)
    assert g.launch()[0] == 0


def _members():
    """Three different contexts: FP64 with buoyancy (istat 3), mixed sweep case
    (istat 2), FP64 with a travelling-wave wall (istat 3)."""
    out = []
    p, x3, jac, inv, var = _strat_case(nP=(24, 16, 21))
    out.append(("fp64_buoy", (p, x3, jac, inv, var), lambda g: g.set_buoyancy(0.5, 1.0)))
    c = sweep_cases(2, grids=[(32, 24, 25), (40, 16, 17)], istat=2)[0]
    out.append(("mixed_sweep", (c.params, c.x3, c.jac, c.inv, c.var), lambda g, c=c: g.set_buoyancy(c.Ri or 0.1, 1.0)))
    p2, x32, jac2, inv2, var2 = make_case(nP=(20, 12, 17), mesh="tanh", beta=2.2, rk=RK3, istat=3, quantize=False)
    wave = W.travelling_wave(0.02, 2.0, 3.0, 0.5)
    out.append(("fp64_wave", (p2, x32, jac2, inv2, var2), lambda g: g.set_wall_bc(0, wave)))
    return out


def _open(spec):
    name, (p, x3, jac, inv, var), setup = spec
    g = Channel(p, x3, jac, inv)
    setup(g)
    g.init_sol_v(var)
    return g


def test_ensemble_matches_members_alone_bit_for_bit():
    specs = _members()
    solo = [_open(s) for s in specs]
    ens_m = [_open(s) for s in specs]
    e = Ensemble(ens_m)
    assert e.block == 6   # lcm(3, 2, 3)
    # 13 = 2 replays + 1 remainder step; then 5 more (remainder only, phase changed);
    # then time averaging on (new graph) and 12 more
    plan = [13, 5, "avg", 12]
    for item in plan:
        if item == "avg":
            for g in solo + ens_m:
                g.time_avg_start()
            continue
        for g in solo:
            g.step(item)
        st = e.step(item)
        assert st == [0, 0, 0]
    replays, captures = e.counters()
    assert replays >= 4 and captures >= 2
    for s, m in zip(solo, ens_m):
        assert np.array_equal(s.download(), m.download())
        assert s.nstep == m.nstep == 30
        assert s.time == m.time
        for a, b in zip(s.stats(), m.stats()):
            assert np.array_equal(a, b)
        ta, tb = s.time_average(), m.time_average()
        assert ta["samples"] == tb["samples"] > 0
        for k in ("mean", "rms", "covar", "tau"):
            assert np.array_equal(ta[k], tb[k]), k
        assert m.debug_canaries() == 0
    e.close()


def test_ensemble_autotuner_leaves_states_unchanged():
    specs = _members()
    a = [_open(s) for s in specs]
    b = [_open(s) for s in specs]
    for g in a:
        g.step(4)
    for g in b:
        g.step(4)
    e = Ensemble(b)
    ms = e.tune(reps=2)
    assert ms > 0
    for sh in e.launch_shapes():
        assert sh[0] in (0, 1, 2, 3) and sh[1] >= 1
    for g in a:
        g.step(8)
    assert e.step(8) == [0, 0, 0]
    for x, y in zip(a, b):
        assert np.array_equal(x.download(), y.download())
        assert x.nstep == y.nstep and x.time == y.time
    e.close()


def test_ensemble_rejects_bad_membership():
    specs = _members()
    g = [_open(s) for s in specs[:2]]
    with pytest.raises(ChanError):
        Ensemble([g[0], g[0]])
    e = Ensemble(g)
    with pytest.raises(ChanError):
        Ensemble([g[1]])              # already in an ensemble
    g[1].diag_enable(planes=(2, 3), every=5)
    with pytest.raises(ChanError):
        e.step(6)                     # members step without the diagnostics series
    e.close()
    e2 = Ensemble([g[1]])             # free again after close
    e2.close()


def test_sweep_ensemble_runs_and_members_stay_finite():
    cases = sweep_cases(4, grids=[(32, 24, 25), (40, 16, 33), (48, 32, 25), (64, 24, 41)])
    chans = [open_case(c) for c in cases]
    e = Ensemble(chans)
    e.tune(reps=1)
    st = e.step(20)
    assert st == [0, 0, 0, 0]
    for c in chans:
        v = c.download()
        assert np.all(np.isfinite(v))
    e.close()


def test_member_blowup_is_reported_for_that_member_only():
    """A member whose dt is far beyond stability blows up (or turns
    non-finite) inside the graph replays; its status says so, and the other
    members still end bit for bit where they end alone."""
    specs = _members()
    good = [_open(s) for s in specs[:2]]
    solo = [_open(s) for s in specs[:2]]
    p, x3, jac, inv, var = specs[2][1]
    bad = Channel(p.with_(dt=p.dt * 400), x3, jac, inv)
    bad.init_sol_v(var)
    e = Ensemble(good + [bad])
    st = e.step(12)
    assert st[0] == 0 and st[1] == 0 and st[2] in (_lib.CHAN_BLOWUP, _lib.CHAN_NONFINITE)
    _, nstep, _ = bad.status_detail()
    assert 1 <= nstep <= 12
    for g in solo:
        g.step(12)
    for a, b in zip(good, solo):
        assert np.array_equal(a.download(), b.download())
    e.close()


# ---------------------------------------------------------------- persistent mode
def _members_of(precision):
    """Two or three contexts of one precision (the persistent kernel runs one
    precision per ensemble): FP64 with buoyancy and FP64 with a travelling
    wave; or two mixed-precision sweep cases of uneven grids."""
    specs = _members()
    if precision == "fp64":
        return [specs[0], specs[2]]
    cs = sweep_cases(3, grids=[(32, 24, 25), (40, 16, 17), (24, 20, 33)], istat=2)
    return [(f"mixed{i}", (c.params, c.x3, c.jac, c.inv, c.var), lambda g, c=c: g.set_buoyancy(c.Ri or 0.1, 1.0))
            for i, c in enumerate(cs)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_ensemble_matches_members_alone(precision):
    """One persistent launch per block: bit for bit the members stepped alone,
    across replays, remainder steps, statistics steps and time averaging."""
    specs = _members_of(precision)
    solo = [_open(s) for s in specs]
    ens_m = [_open(s) for s in specs]
    e = Ensemble(ens_m)
    e.set_mode("persistent")
    plan = [13, 5, "avg", 12]
    for item in plan:
        if item == "avg":
            for g in solo + ens_m:
                g.time_avg_start()
            continue
        for g in solo:
            g.step(item)
        assert e.step(item) == [0] * len(specs)
        assert e.mode_in_use() == ("persistent", "")
    for s, m in zip(solo, ens_m):
        assert np.array_equal(s.download(), m.download())
        assert s.nstep == m.nstep and s.time == m.time
        for a, b in zip(s.stats(), m.stats()):
            assert np.array_equal(a, b)
        ta, tb = s.time_average(), m.time_average()
        assert ta["samples"] == tb["samples"] > 0
        for k in ("mean", "rms", "covar", "tau"):
            assert np.array_equal(ta[k], tb[k]), k
        assert m.debug_canaries() == 0
    e.close()


def test_persistent_mode_falls_back_for_mixed_precisions_and_graph_mode_matches():
    specs = _members()            # FP64 and mixed members together
    e = Ensemble([_open(s) for s in specs])
    e.set_mode("persistent")
    e.step(6)
    assert e.mode_in_use() == ("graph", "members of both precisions")
    e.close()
    fp = _members_of("fp64")
    a = [_open(s) for s in fp]
    b = [_open(s) for s in fp]
    ea, eb = Ensemble(a), Ensemble(b)
    ea.set_mode("persistent")
    ea.step(12)
    eb.step(12)
    assert ea.mode_in_use()[0] == "persistent" and eb.mode_in_use()[0] == "graph"
    for x, y in zip(a, b):
        assert np.array_equal(x.download(), y.download())
    ea.close()
    eb.close()


def test_persistent_dependency_wait_gives_up_and_reports():
    """Host-side fault injection: member 0's first stage waits for work that
    never completes.  The bounded waits end the launch with CHAN_ECUDA within
    seconds (no hang), and after a fresh upload the ensemble runs correctly."""
    import time
    specs = _members_of("fp64")
    ens_m = [_open(s) for s in specs]
    e = Ensemble(ens_m)
    e.set_mode("persistent-stall-test")
    t0 = time.time()
    with pytest.raises(ChanError) as ei:
        e.step(e.block)
    assert ei.value.code == _lib.CHAN_ECUDA and "waited more than a second" in str(ei.value)
    assert time.time() - t0 < 30
    e.set_mode("persistent")
    solo = [_open(s) for s in specs]
    for g, s in zip(ens_m, specs):
        g.init_sol_v(s[1][4])
    for g in solo:
        g.step(6)
    assert e.step(6) == [0, 0]
    for x, y in zip(solo, ens_m):
        assert np.array_equal(x.download(), y.download())
    e.close()


def test_persistent_member_blowup_is_reported_for_that_member_only():
    specs = _members_of("fp64")
    good = [_open(specs[0])]
    solo = [_open(specs[0])]
    p, x3, jac, inv, var = specs[1][1]
    bad = Channel(p.with_(dt=p.dt * 400), x3, jac, inv)
    bad.init_sol_v(var)
    e = Ensemble(good + [bad])
    e.set_mode("persistent")
    st = e.step(12)
    assert e.mode_in_use()[0] == "persistent"
    assert st[0] == 0 and st[1] in (_lib.CHAN_BLOWUP, _lib.CHAN_NONFINITE)
    solo[0].step(12)
    assert np.array_equal(good[0].download(), solo[0].download())
    e.close()
