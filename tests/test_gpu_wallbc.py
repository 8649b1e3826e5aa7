"""Wall-BC plug-ins of the sm_100a library against the oracle.

Each reference wall variant (v1.9_strat st1-st4, v1.9_groov g1,
v1.9_groov_strat gst1-gst5, v1.9_STWNV s1-s6, v1.9_RD rd1-rd3) is set on the
bottom wall of both sides and stepped; the fields must agree to <= 1e-12
relative per step (same metric as the other parity tests), and the wall shear
and plane moments that feed the forcing to <= 1e-12 of their scale.
"""
import numpy as np
import pytest

from chan_cases import CASES, make_case, rel_err, worst
from compchan3dmpi_b200 import Channel, ChanError, RK3
from compchan3dmpi_b200 import wallbc as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12

VARIANTS = ["st1", "st2", "st3", "st4", "g1", "gst2", "gst3", "gst5", "s1", "s3", "s4", "s5", "rd1", "rd3"]


def _pair(case, bottom, top=None):
    p, x3, jac, inv, var = case
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    g.set_wall_bc(0, bottom)
    o.set_wall_bc(0, bottom)
    if top is not None:
        g.set_wall_bc(1, top)
        o.set_wall_bc(1, top)
    return g, o


@pytest.mark.parametrize("name", VARIANTS)
def test_reference_variant(name):
    case = make_case(**CASES["ref_rk2_cosine"])
    bottom, top = W.reference_variant(name, case[0])
    g, o = _pair(case, bottom, top)
    for s in range(1, 5):
        g.step(1)
        o.step(1)
        gv, ov = g.download(), o.download()
        e = rel_err(gv, ov)
        assert e.max() <= TOL, f"{name} step {s}: {e} worst at {worst(gv, ov)}"
    gt, g1, g2, gc = g.stats()
    ot, o1, o2, oc = o.stats()
    assert np.all(np.abs(gt - ot) <= TOL * np.max(np.abs(ot))), (gt, ot)
    for a, b in ((g1, o1), (g2, o2), (gc, oc)):
        assert np.max(np.abs(a - b)) <= TOL * max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", ["st3", "gst2", "s3", "rd1"])
def test_variant_rk3_tanh_both_walls(name):
    """Production physics (RK3, tanh mesh) with the variant on both walls."""
    case = make_case(**CASES["rk3_tanh"])
    bottom, _ = W.reference_variant(name, case[0])
    g, o = _pair(case, bottom, bottom)
    for s in range(1, 4):
        g.step(1)
        o.step(1)
        gv, ov = g.download(), o.download()
        e = rel_err(gv, ov)
        assert e.max() <= TOL, f"{name} step {s}: {e} worst at {worst(gv, ov)}"


def test_single_stage_wave_time():
    """A stage run alone sees the next step's time in the wave (as step() does)."""
    case = make_case(**CASES["ragged"])
    bottom, _ = W.reference_variant("s1", case[0])
    g, o = _pair(case, bottom)
    g.stage(1)
    o.stage(1)
    gv, ov = g.download(), o.download()
    assert rel_err(gv, ov).max() <= TOL


def test_wall_bc_errors():
    case = make_case(**CASES["ragged"])
    p, x3, jac, inv, var = case
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    with pytest.raises(ChanError):
        g.set_wall_bc(0, W.WallBC(velocity=W.SLIP_MASK))     # no mask
    with pytest.raises(ChanError):
        g.set_wall_bc(0, W.WallBC(velocity=W.UV_FIELD))      # no uv
    with pytest.raises(ChanError):
        g.set_wall_bc(2, W.isothermal(1.0))                  # no such wall
    with pytest.raises(ChanError):
        g.set_wall_bc(0, W.isothermal(-1.0))
    with pytest.raises(ChanError):
        g.set_wall_bc(0, W.WallBC(velocity=7))


@pytest.mark.parametrize("name", ["st4", "gst2", "s3", "rd1"])
def test_variant_40_steps_with_forcing(name):
    """Longer runs with the lagged forcing refreshed every 5 steps: no drift."""
    case = make_case(nP=(24, 16, 21), mesh="tanh", beta=2.0, rk=RK3, Pr=0.72, istat=5, quantize=False)
    bottom, top = W.reference_variant(name, case[0])
    g, o = _pair(case, bottom, top)
    for blk in range(4):
        g.step(10)
        o.step(10)
        gv, ov = g.download(), o.download()
        e = rel_err(gv, ov)
        assert e.max() <= TOL, f"{name} step {10 * (blk + 1)}: {e} worst at {worst(gv, ov)}"


def test_checkpoint_restart_with_wall_bc(tmp_path):
    """The checkpoint holds the state, not the wall-BC setting: restore, set the BC
    again, and the run continues bit for bit."""
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), quantize=False, istat=3)
    bottom, top = W.reference_variant("gst5", p)
    a = Channel(p, x3, jac, inv)
    a.init_sol_v(var)
    a.set_wall_bc(0, bottom)
    a.step(8)
    ref = a.download()
    b = Channel(p, x3, jac, inv)
    b.init_sol_v(var)
    b.set_wall_bc(0, bottom)
    b.step(4)
    b.checkpoint_write(tmp_path / "w.ckp")
    c = Channel(p, x3, jac, inv)
    c.set_wall_bc(0, bottom)
    c.checkpoint_read(tmp_path / "w.ckp")
    c.step(4)
    assert np.array_equal(c.download(), ref)
