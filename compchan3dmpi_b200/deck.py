"""Input decks in the reference's own formats.

* ``param.dat``: fixed-column run deck.  Values start at column 49 ('48X' in
  every read format), v1.9/codes/comdata.f90:31-68.
* ``3D.dat``: Tecplot-ASCII POINT restart/output file.
  Header ``TITLE ="<time F20.10><nstep I9>"``, a ``Variables=`` line and a
  ``ZONE`` line.  Then k, j, i loops with one blank line before each k and
  each j block.  Records are ``3(1X,F10.6),7(1X,E22.15)``: x,y,z,rho,u,v,w,E,T,p
  (writer v1.9/codes/main_v1.9.f90:759-773, reader :213-239).

Fields use the layout ``var[m, k, j, i]`` (Fortran var(1:nP1,1:nP2,1:nP3,1:7)).
Parse errors raise ``DeckError`` naming the offending record, as the
reference prints "Error in reading combined input file at i j k".
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

from .params import ChanParams


class DeckError(ValueError):
    pass


# ------------------------------------------------------------------ E22.15
def fmt_e(x: float, w: int, d: int) -> str:
    """Fortran Ew.d output: [-]0.<d digits>E+xx, right-justified in w columns
    (3-digit exponents drop the letter: 0.123+100)."""
    if x != x or math.isinf(x):
        return ("NaN" if x != x else ("-Infinity" if x < 0 else "Infinity")).rjust(w)
    neg = math.copysign(1.0, x) < 0 and x != 0.0
    if x == 0.0:
        body = "0." + "0" * d + "E+00"
    else:
        s = f"{abs(x):.{d - 1}E}"
        mant, ex = s.split("E")
        digits = mant.replace(".", "")
        e = int(ex) + 1
        body = f"0.{digits}E{e:+03d}" if abs(e) <= 99 else f"0.{digits}{e:+04d}"
    out = ("-" if neg else "") + body
    return out.rjust(w) if len(out) <= w else "*" * w


def fmt_e22_15(x: float) -> str:
    """Fortran E22.15 output: 0.ddddddddddddddd E+xx, right-justified to 22."""
    return fmt_e(x, 22, 15)


def parse_fortran_real(s: str) -> float:
    s = s.strip()
    if not s:
        return 0.0
    t = s.replace("D", "E").replace("d", "e")
    try:
        return float(t)
    except ValueError:
        pass
    # exponent without a letter, e.g. 0.123+100
    for pos in range(len(t) - 1, 0, -1):
        if t[pos] in "+-" and t[pos - 1].isdigit():
            return float(t[:pos] + "E" + t[pos:])
    raise DeckError(f"bad real field {s!r}")


def quantize_deck(var: np.ndarray) -> np.ndarray:
    """Round every value to what an E22.15 record holds (15 significant digits)."""
    flat = np.asarray(var, dtype=np.float64).ravel()
    out = np.fromiter((parse_fortran_real(fmt_e22_15(float(v))) for v in flat), dtype=np.float64,
                      count=flat.size)
    return out.reshape(np.shape(var))


# ----------------------------------------------------------------- param.dat
_PARAM_LINES = [
    ("skip", None), ("skip", None),
    ("descp", "A"), ("resOp", "i1"), ("skip", None),
    ("topo1", "i2"), ("topo2", "i2"), ("topo3", "i2"), ("skip", None), ("skip", None),
    ("Re", "F4.0"), ("Mac", "f3.1"), ("dt", "f6.4"), ("istat", "i2"), ("skip", None),
    ("PexVal", "f3.1"), ("PeyVal", "f3.1"), ("PezVal", "f3.1"), ("skip", None),
    ("debugOp", "i1"), ("inputPath", "A"),
]

_LABELS = {
    "descp": "Case Description", "resOp": "Restart Option [1/2]", "topo1": "MPI processes in x",
    "topo2": "MPI processes in y", "topo3": "MPI processes in z", "Re": "Reynolds Number",
    "Mac": "Mach Number", "dt": "Timestep", "istat": "Freq of stat calculation",
    "PexVal": "Peclet in x-direction", "PeyVal": "Peclet in y-direction",
    "PezVal": "Peclet in z-direction", "debugOp": "Debug Option [0/1]", "inputPath": "Path to input file",
}


def _width(fmt: str) -> int:
    return int("".join(ch for ch in fmt[1:].split(".")[0] if ch.isdigit()))


def _read_field(line: str, fmt: str):
    field = line[48:]
    if fmt == "A":
        return field.rstrip("\n").strip()
    w = _width(fmt)
    raw = field[:w]
    if fmt[0] in "iI":
        return int(raw.strip() or "0")
    # F editing: with no decimal point the last d digits are decimals
    d = int(fmt.split(".")[1])
    txt = raw.strip()
    if not txt:
        return 0.0
    if "." in txt or "e" in txt.lower() or "d" in txt.lower():
        return parse_fortran_real(txt)
    return int(txt) / 10.0 ** d


def _fmt_field(val, fmt: str) -> str:
    if fmt == "A":
        return str(val)
    w = _width(fmt)
    if fmt[0] in "iI":
        s = f"{int(val):{w}d}"
    else:
        d = int(fmt.split(".")[1])
        s = f"{float(val):{w}.{d}f}"
        if len(s) > w or abs(float(s) - float(val)) > 1e-12 * max(1.0, abs(float(val))):
            # not representable in Fw.d: Fortran F input also accepts an exponent
            for p in range(w, 0, -1):
                t = f"{float(val):.{p}e}".replace("e-0", "e-").replace("e+0", "e+")
                if len(t) <= w:
                    s = t.rjust(w)
                    break
    if len(s) > w:
        raise DeckError(f"value {val!r} does not fit format {fmt}")
    return s


def write_param_dat(path, params: ChanParams, descp="compChan", resOp=1, topo=(1, 1, 1), debugOp=0,
                    inputPath="3D.dat"):
    vals = {"descp": descp, "resOp": resOp, "topo1": topo[0], "topo2": topo[1], "topo3": topo[2],
            "Re": params.Re, "Mac": params.Mac, "dt": params.dt, "istat": params.istat,
            "PexVal": params.Pe[0], "PeyVal": params.Pe[1], "PezVal": params.Pe[2],
            "debugOp": debugOp, "inputPath": inputPath}
    lines = []
    for n, (name, fmt) in enumerate(_PARAM_LINES):
        if name == "skip":
            lines.append("=" * 60 if n in (0, 1) else "-" * 60)
            continue
        label = _LABELS[name].ljust(46)[:46] + ": "
        lines.append(label + _fmt_field(vals[name], fmt))
    Path(path).write_text("\n".join(lines) + "\n")


def read_param_dat(path, nP=(64, 48, 65), **kw):
    """Returns (ChanParams, extras) where extras holds descp, resOp, topo, debugOp, inputPath."""
    lines = Path(path).read_text().splitlines()
    if len(lines) < len(_PARAM_LINES):
        raise DeckError(f"{path}: {len(lines)} lines, expected {len(_PARAM_LINES)}")
    vals = {}
    for n, (name, fmt) in enumerate(_PARAM_LINES):
        if name == "skip":
            continue
        try:
            vals[name] = _read_field(lines[n], fmt)
        except (ValueError, IndexError) as e:
            raise DeckError(f"{path}: line {n + 1} ({name}): {e}") from None
    p = ChanParams(nP=tuple(nP), Re=float(vals["Re"]), Mac=float(vals["Mac"]), dt=float(vals["dt"]),
                   istat=int(vals["istat"]), Pe=(float(vals["PexVal"]), float(vals["PeyVal"]), float(vals["PezVal"])),
                   **kw)
    extras = {k: vals[k] for k in ("descp", "resOp", "debugOp", "inputPath")}
    extras["topo"] = (vals["topo1"], vals["topo2"], vals["topo3"])
    return p, extras


# ------------------------------------------------------------------- 3D.dat
def write_3d_dat(path, var: np.ndarray, x1, x2, x3, time: float = 0.0, nstep: int = 0):
    _, n3, n2, n1 = var.shape
    out = [f'TITLE ="{time:20.10f}{nstep:9d}"',
           ' Variables ="x","y","z","Rho","U","V","W","E","T","P"',
           f"ZONE k={n3:3d},j={n2:3d},i={n1:3d},DATAPACKING=\"POINT\""]
    for k in range(n3):
        out.append("")
        for j in range(n2):
            out.append("")
            for i in range(n1):
                rec = f" {x1[i]:10.6f} {x2[j]:10.6f} {x3[k]:10.6f}" + "".join(
                    " " + fmt_e22_15(float(var[m, k, j, i])) for m in range(7))
                out.append(rec)
    Path(path).write_text("\n".join(out) + "\n")


def read_3d_dat(path, nP):
    """Returns var (7,nP3,nP2,nP1), time, nstep, x1, x2, x3."""
    n1, n2, n3 = nP
    with open(path) as f:
        head = f.readline()
        try:
            time = float(head[8:28])
            nstep = int(head[28:37])
        except ValueError:
            raise DeckError(f"{path}: bad header {head!r}") from None
        f.readline()
        f.readline()
        var = np.empty((7, n3, n2, n1))
        x1 = np.empty(n1); x2 = np.empty(n2); x3 = np.empty(n3)
        for k in range(n3):
            f.readline()
            for j in range(n2):
                f.readline()
                for i in range(n1):
                    line = f.readline()
                    if len(line.rstrip("\n")) < 33 + 7 * 23:
                        raise DeckError(f"Error in reading combined input file at {i + 1} {j + 1} {k + 1}")
                    try:
                        x1[i] = float(line[1:11]); x2[j] = float(line[12:22]); x3[k] = float(line[23:33])
                        for m in range(7):
                            a = 33 + m * 23 + 1
                            var[m, k, j, i] = parse_fortran_real(line[a:a + 22])
                    except (ValueError, DeckError):
                        raise DeckError(f"Error in reading combined input file at {i + 1} {j + 1} {k + 1}") from None
    return var, time, nstep, x1, x2, x3


# ------------------------------------------------- native (library) versions
def _native():
    from . import _lib
    return _lib.load()


def write_3d_dat_native(path, var, x1, x2, x3, time=0.0, nstep=0, threads=0):
    """Same bytes as write_3d_dat, formatted on host threads by the library."""
    import ctypes
    from . import _lib
    L = _native()
    v = np.ascontiguousarray(var, dtype=np.float64)
    _, n3, n2, n1 = v.shape
    nP = (ctypes.c_int32 * 3)(n1, n2, n3)
    a1, a2, a3 = (np.ascontiguousarray(a, dtype=np.float64) for a in (x1, x2, x3))
    r = L.chan_deck_write(str(path).encode(), nP, _lib.dptr(v), _lib.dptr(a1), _lib.dptr(a2), _lib.dptr(a3),
                          float(time), int(nstep), int(threads))
    if r != 0:
        raise DeckError(L.chan_io_last_error().decode())


def read_3d_dat_native(path, nP, threads=0):
    """Same result as read_3d_dat, parsed on host threads by the library."""
    import ctypes
    from . import _lib
    L = _native()
    n1, n2, n3 = nP
    var = np.empty((7, n3, n2, n1))
    x1 = np.empty(n1); x2 = np.empty(n2); x3 = np.empty(n3)
    t = ctypes.c_double(); n = ctypes.c_int64()
    nPc = (ctypes.c_int32 * 3)(n1, n2, n3)
    r = L.chan_deck_read(str(path).encode(), nPc, _lib.dptr(var), _lib.dptr(x1), _lib.dptr(x2), _lib.dptr(x3),
                         ctypes.byref(t), ctypes.byref(n), int(threads))
    if r != 0:
        raise DeckError(L.chan_io_last_error().decode())
    return var, t.value, n.value, x1, x2, x3
