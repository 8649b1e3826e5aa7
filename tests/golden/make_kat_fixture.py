"""Extract the reference's own known-answer test output into a fixture.

The serial reference code applies its one-sided wall coefficients to
p(x) = x^3 - 5x^2 + 3x - 10 on the nP3=160 cosine mesh and prints the result
next to the exact derivative
(v1.8_validation/codes/mainV1.8_serial.f90:76-105, 808-824).  The captured
output is v1.8_validation/codes/nohupDebug.out:23-26.

Run where the reference is checked out, giving its root directory:
    python tests/golden/make_kat_fixture.py <reference-root>
"""
import json
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit("usage: make_kat_fixture.py <reference-root>")
ref = Path(sys.argv[1])
lines = (ref / "v1.8_validation/codes/nohupDebug.out").read_text().splitlines()
rows = {}
for ln in lines[22:26]:
    label, nums = ln.split(":")
    got, exact = (float(t) for t in nums.split())
    rows[label.strip()] = {"logged": got, "exact": exact}
out = {
    "source": "v1.8_validation/codes/nohupDebug.out:23-26",
    "code": "v1.8_validation/codes/mainV1.8_serial.f90:76-105",
    "mesh": {"kind": "cosine", "nP3": 160},
    "polynomial": "x**3 - 5*x**2 + 3*x - 10",
    "rows": rows,
}
Path(__file__).with_name("fd_coeff_kat.json").write_text(json.dumps(out, indent=1) + "\n")
print(json.dumps(out, indent=1))
