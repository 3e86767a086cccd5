"""Copy the reference's inverse-Hopf product-grid fixture into hopf.npz.

Run once, in a checkout where the reference project is available:

    python tests/golden/make_hopf.py /path/to/reference

The reference's tests/fixtures/hopf-reference.npz holds SO3K_Grids
`so3k.product.product_grid(group, f)` in float64 for all eleven groups at small
frequencies (the rows src/hopf.zig must reproduce, compared orbit by orbit in
tests/test_hopf.py:42-54). The grid rows are stored unchanged under their own keys
(`<group>_<f>`); the covering bounds belong to the covering measures, which this engine
does not build, and are left out.
"""
import sys
from pathlib import Path

import numpy as np


def main(root):
    src = Path(root) / "tests" / "fixtures" / "hopf-reference.npz"
    with np.load(src) as data:
        rows = {k: data[k] for k in data.files if not k.endswith("_bound")}
    out = Path(__file__).resolve().parent / "hopf.npz"
    np.savez_compressed(out, **rows)
    print(f"wrote {out}: {len(rows)} grids, {sum(len(v) for v in rows.values())} rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_hopf.py <reference checkout>")
    main(sys.argv[1])
