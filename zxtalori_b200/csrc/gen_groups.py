"""Generate groups_table.inc: the eleven proper point groups' operator quaternions.

The engine's symmetry tables must equal the reference's bit for bit (zo_operations
returns them, image order fixes shell codes and fold tie-breaking), so they are not
re-derived: they are read from the reference's published operator fixture
(tests/fixtures/pair-operators.npz, which equals src/groups.zig:39-201 value for value)
and written out as exact hexadecimal float literals, f64 and the f32 rounding the
reference uploads (src/groups.zig:24-38, "f64 literals cast to f32").

Run once where the reference checkout exists:
    python zxtalori_b200/csrc/gen_groups.py <reference>/tests/fixtures/pair-operators.npz
The generated file is committed; nothing reads the reference at build or run time.
"""
import sys
from pathlib import Path

import numpy as np

GROUPS = ("C2", "C3", "C4", "C6", "D2", "D3", "D4", "D6", "T", "O", "I")


def main(path):
    data = np.load(path)
    out = ["// Generated by gen_groups.py from the reference's operator fixture; do not edit.",
           "// Scalar-first unit quaternions, right action q*g; row 0 is the identity.",
           "// clang-format off"]
    offsets, total = [], 0
    f64_rows, f32_rows = [], []
    for g in GROUPS:
        ops = np.asarray(data[g], dtype=np.float64)
        offsets.append((g, total, len(ops)))
        total += len(ops)
        for row in ops:
            f64_rows.append(", ".join(float(v).hex() for v in row))
            f32_rows.append(", ".join(float(np.float32(v)).hex() + "f" for v in row))
    out.append(f"static const int kGroupCount = {len(GROUPS)};")
    out.append(f"static const int kOperatorRows = {total};")
    out.append("static const int kGroupOffset[11] = {" + ", ".join(str(o) for _, o, _ in offsets) + "};")
    out.append("static const int kGroupOrder[11] = {" + ", ".join(str(n) for _, _, n in offsets) + "};")
    out.append("static const char* const kGroupName[11] = {" + ", ".join(f'"{g}"' for g in GROUPS) + "};")
    out.append("static const double kOps64[%d][4] = {" % total)
    out += ["  {" + r + "}," for r in f64_rows]
    out.append("};")
    out.append("static const float kOps32[%d][4] = {" % total)
    out += ["  {" + r + "}," for r in f32_rows]
    out.append("};")
    out.append("// clang-format on")
    target = Path(__file__).resolve().parent / "groups_table.inc"
    target.write_text("\n".join(out) + "\n")
    print("wrote", target, total, "rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: gen_groups.py <reference checkout>/tests/fixtures/pair-operators.npz")
    main(sys.argv[1])
