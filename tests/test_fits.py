"""The device arithmetic's polynomial tables (qvm_device.cuh) are the ones fit_atan.py
reproduces, and meet their stated relative-error bounds with their float32 coefficients:
the arctangent over t in [0, 1] (6.4e-8, about one float ulp) and [0, 0.21] (6.0e-9), and
the short-chord angle and sine over d in [0, 0.25] (below 1e-8)."""
import re
import sys
from pathlib import Path

import numpy as np
import pytest

CSRC = Path(__file__).resolve().parents[1] / "zxtalori_b200" / "csrc"
sys.path.insert(0, str(CSRC))
import fit_atan  # noqa: E402

HEADER = (CSRC / "qvm_device.cuh").read_text()
HEX = re.compile(r"-?0x1\.[0-9a-f]+p[-+]?\d+f")


def body(name):
    start = HEADER.index(name + "(")
    return HEADER[start:HEADER.index("\n}\n", start)]


def literals(text):
    return [float.fromhex(h[:-1]) for h in HEX.findall(text)]


def f32(v):
    return float(np.float32(v))


@pytest.mark.parametrize("name,degree,t_max,bound", [("two_atan_unit", 8, 1.0, 6.5e-8),
                                                     ("two_atan_short", 3, 0.21, 6.1e-9)])
def test_arctangent_tables(name, degree, t_max, bound):
    # Horner from the highest power down to the constant 2 (not written in hex).
    table = literals(body(name))[::-1]
    coeffs, _ = fit_atan.fit(degree, t_max=t_max)
    assert table == [f32(2 * c) for c in coeffs[1:]]
    assert f32(2 * coeffs[0]) == 2.0
    c = np.array([2.0] + table)
    t = np.linspace(1e-6, t_max, 200_001)
    approx = t * np.polyval(c[::-1], t * t)
    assert np.max(np.abs(approx / (2 * np.arctan(t)) - 1)) < bound


def test_chord_tables():
    text = body("near_chord_pair32x2")
    pa_line = next(line for line in text.splitlines() if "const float2 pa" in line)
    ps_line = next(line for line in text.splitlines() if "const float2 ps" in line)
    pa, ps = literals(pa_line)[::-1], literals(ps_line)[::-1]  # written highest power first
    for table, target in ((pa, fit_atan.chord_angle), (ps, fit_atan.chord_sine)):
        coeffs, _ = fit_atan.fit_chord(target)
        assert table == [f32(c) for c in coeffs]
        d = np.linspace(1e-9, 0.25, 200_001)
        approx = 1 + d * np.polyval(np.array(table)[::-1], d)
        assert np.max(np.abs(approx / target(d) - 1)) < 1e-8
