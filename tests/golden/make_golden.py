"""Generate the golden vectors that pin the oracle to the reference's own dense models.

Run once, in a checkout where the reference project is available:

    python tests/golden/make_golden.py /path/to/reference

It imports the reference's pure-NumPy test models with the GPU-only `wgpu` module stubbed
(nothing of the reference's engine runs):
  * tests/test_pair_kernels.py:27-69   reference(q, ops)      -> dense FP64 per-source rows
  * tests/test_measures.py:198-213      expected_measures(q, ops)
  * tests/test_near_field.py:14-40      mean_radius(count), near_reference(q, ops, delta)
and records inputs and outputs in golden.npz, together with the operator table fixture
(tests/fixtures/pair-operators.npz, the reference's f64 group tables). The committed
golden.npz is what the tests read; nothing reads the reference at test time.
"""
import importlib
import math
import sys
import types
from pathlib import Path

import numpy as np

GROUPS = ("C2", "C3", "C4", "C6", "D2", "D3", "D4", "D6", "T", "O", "I")


def load_reference(root):
    sys.modules.setdefault("wgpu", types.ModuleType("wgpu"))
    sys.path.insert(0, str(root / "python"))
    sys.path.insert(0, str(root / "tests"))
    kernels = importlib.import_module("test_pair_kernels")
    measures = importlib.import_module("test_measures")
    near = importlib.import_module("test_near_field")
    return kernels, measures, near


def main(root):
    root = Path(root)
    kernels, measures, near = load_reference(root)
    fixture = np.load(root / "tests/fixtures/pair-operators.npz")
    out = {}
    for g in GROUPS:
        out[f"ops_{g}"] = np.asarray(fixture[g], np.float64)

    # Dense rows, the reference's own input recipe (test_pair_kernels.py:118-119).
    rng = np.random.default_rng(752)
    q = rng.normal(size=(37, 4))
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    q = q.astype(np.float32)
    out["rows_q"] = q
    for g in GROUPS:
        ops32 = np.asarray(fixture[g], np.float32)
        out[f"rows_{g}"] = kernels.reference(q, ops32)
    # Antipodal sign changes (test_pair_kernels.py:132) must leave rows unchanged.
    signed = q.copy()
    signed[::2] *= -1
    out["rows_signed_q"] = signed
    out["rows_signed_O"] = kernels.reference(signed, np.asarray(fixture["O"], np.float32))

    # Measures (test_measures.py:217-218).
    rng = np.random.default_rng(312)
    q = rng.normal(size=(29, 4))
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    out["measures_q"] = q
    keys = ("riesz_1", "riesz_2", "riesz_3", "green_ratio", "log_ratio", "quey_energy", "separation_deg", "force_rms")
    out["measures_keys"] = np.array(keys)
    for g in GROUPS:
        m = measures.expected_measures(q, np.asarray(fixture[g], np.float32))
        out[f"measures_{g}"] = np.array([m[k] for k in keys])
    # A near pair at 5e-5 rad resolved through chords (test_measures.py:249-255).
    pair = np.array([[1, 0, 0, 0], [math.cos(5e-5), math.sin(5e-5), 0, 0]], np.float64)
    out["near_pair_q"] = pair
    m = measures.expected_measures(pair, np.asarray(fixture["C2"], np.float32))
    out["near_pair_measures"] = np.array([m[k] for k in keys])

    # Mean orientation radius (src/pairs.zig:205-215 as restated by the test).
    counts = np.array([2, 48, 1000, 25152, 2_400_000, 60_000_000, 600_000_000], np.int64)
    out["radius_counts"] = counts
    out["radius_values"] = np.array([near.mean_radius(int(c)) for c in counts])

    # Windowed near-field energy and separation (test_near_field.py:23-40).
    for g, n, seed in (("O", 300, 11), ("D6", 240, 12), ("C2", 200, 13), ("I", 120, 14)):
        rng = np.random.default_rng(seed)
        q = rng.normal(size=(n, 4))
        q /= np.linalg.norm(q, axis=-1, keepdims=True)
        ops = np.asarray(fixture[g], np.float32)
        energy, sep = near.near_reference(q, ops, 20)
        out[f"near_{g}_q"] = q
        out[f"near_{g}"] = np.array([energy, sep, 20.0])

    target = Path(__file__).resolve().parent / "golden.npz"
    np.savez_compressed(target, **out)
    print("wrote", target, len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    main(sys.argv[1])
