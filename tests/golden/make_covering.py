"""Copy the reference's published covering radii, and the grids they were measured on, into
covering.npz.

Run once, in a checkout where the reference project is available:

    python tests/golden/make_covering.py /path/to/reference

The reference's tests/fixtures/covering-reference.json records, per group, the covering
radius (SO(3) degrees) of a small grid: for the cyclic and dihedral groups the inverse-Hopf
product grid at frequency 2 (rows in tests/fixtures/hopf-reference.npz, copied here as
hopf.npz), for T, O and I the h=2 grids of tests/fixtures/reference-small.npz (copied
here). C6's entry (52 rows) matches neither fixture and is left out. Stored: `<group>_rows`
(T, O, I), `<group>_grid` (the hopf.npz key, C/D groups) and `<group>_radius_deg`.
"""
import json
import sys
from pathlib import Path

import numpy as np

HOPF_KEYS = {"C2": "C2_2", "C3": "C3_2", "C4": "C4_2", "D2": "D2_2", "D3": "D3_2", "D4": "D4_2", "D6": "D6_2"}


def main(root):
    fixtures = Path(root) / "tests" / "fixtures"
    radii = json.loads((fixtures / "covering-reference.json").read_text())
    out = {}
    with np.load(fixtures / "reference-small.npz") as small, np.load(fixtures / "hopf-reference.npz") as hopf:
        for group, entry in radii.items():
            if group in HOPF_KEYS:
                key = HOPF_KEYS[group]
                assert hopf[key].shape[0] == entry["count"], (group, key)
                out[f"{group}_grid"] = np.array(key)
            elif group in ("T", "O", "I"):
                assert small[group].shape[0] == entry["count"], group
                out[f"{group}_rows"] = small[group]
            else:
                continue
            out[f"{group}_radius_deg"] = np.float64(entry["radius_deg"])
    dest = Path(__file__).resolve().parent / "covering.npz"
    np.savez_compressed(dest, **out)
    print(f"wrote {dest}: {sorted(k for k in out if k.endswith('_radius_deg'))}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_covering.py <reference checkout>")
    main(sys.argv[1])
