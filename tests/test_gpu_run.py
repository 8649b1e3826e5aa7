"""The reference's time loop driver (compchan3dmpi_b200.run) end to end: run
deck in, output series and restart decks out, blow-up dump."""
import numpy as np
import pytest

from chan_cases import make_case
from compchan3dmpi_b200 import periodic_coords
from compchan3dmpi_b200.deck import read_3d_dat, write_3d_dat, write_param_dat
from compchan3dmpi_b200.run import run
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _case_dir(tmp_path, var, p, x3):
    (tmp_path / "codes").mkdir()
    (tmp_path / "input").mkdir()
    write_param_dat(tmp_path / "param.dat", p, inputPath="../input/3D.dat")
    write_3d_dat(tmp_path / "input" / "3D.dat", var, periodic_coords(p.nP[0], p.Lx),
                 periodic_coords(p.nP[1], p.Ly), x3, 0.0, 0)
    return tmp_path


def test_driver_outputs_and_restart_deck(tmp_path):
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), istat=5, dt=1e-3)
    d = _case_dir(tmp_path, var, p, x3)
    lines = []
    assert run(d, p.nP, maxstep=1000, log=lines.append) == 0
    out = d / "output"
    assert len((out / "KE.dat").read_text().splitlines()) == 100
    assert len((out / "massflow.dat").read_text().splitlines()) == 100
    assert len((out / "tauWall.dat").read_text().splitlines()) == 200
    assert len((out / "moment1st.dat").read_text().splitlines()) == 200
    assert len([ln for ln in lines if "CPU Time" in ln]) == 100
    # step 1000 is an odd multiple of 1000: the alternate restart deck
    back, t, n, *_ = read_3d_dat(out / "3D001_.dat", p.nP)
    assert n == 1000 and abs(t - 1000 * p.dt) < 1e-9
    o = O.Oracle(p, x3, jac, inv)
    o.upload(read_3d_dat(d / "input" / "3D.dat", p.nP)[0])
    o.step(1000)
    ov = o.download()
    e = max(np.max(np.abs(back[m] - ov[m])) / np.max(np.abs(ov[m])) for m in range(7))
    assert e <= 1e-11, e
    # restart from the written deck (resOp = 2 reads output/3D001.dat)
    (out / "3D001.dat").write_bytes((out / "3D001_.dat").read_bytes())
    write_param_dat(d / "param.dat", p, resOp=2, inputPath="../input/3D.dat")
    assert run(d, p.nP, maxstep=1010, log=lines.append) == 0
    assert len((out / "KE.dat").read_text().splitlines()) == 101


def test_driver_blowup_dump(tmp_path):
    p, x3, jac, inv, var = make_case(nP=(20, 14, 19), istat=5, quantize=False)
    var = var.copy()
    var[0, 6, 5, 7] = -1.0
    d = _case_dir(tmp_path, var, p, x3)
    lines = []
    assert run(d, p.nP, maxstep=50, log=lines.append) == 1
    assert (d / "debug" / "3D001.dat").exists()
    rec = (d / "debug" / "3D001.dat").read_text().splitlines()[5]
    assert len(rec) == 3 * 8 + 7 * 13
    assert len(lines) == 1 and len(lines[0]) == 10 + 4 * 4 + 2 * 8
