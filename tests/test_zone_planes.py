"""The zone bisector planes' reach (no GPU): the shell's rim test takes the planes in order of
reach and stops at the first whose reach exceeds the shell margin, so each reach must bound
the plane's dot product below over the whole zone. Checked against the oracle's fold of
200,000 Haar orientations per group, and against the zone's own faces (the planes that
touch the zone come first, with reach -1)."""
import ctypes as C

import numpy as np
import pytest

from conftest import GROUPS
from oracle import qvm

FACES = {"D2": 6, "D3": 8, "D4": 10, "D6": 14, "T": 14, "O": 14, "I": 12}


def planes_of(ops):
    """The reference's plane list (src/covering.zig:382-396): e - s g_k, normalised, for each
    operator and sign but (identity, +1)."""
    rows = []
    for k in range(len(ops)):
        for s in (1.0, -1.0):
            if k == 0 and s == 1.0:
                continue
            v = np.array([1.0, 0, 0, 0]) - s * ops[k]
            rows.append(v / np.linalg.norm(v))
    return np.array(rows)


@pytest.fixture(scope="module")
def zone_planes():
    from zxtalori_b200 import build

    lib = C.CDLL(str(build.build(verbose=False)))
    lib.zo_zone_planes.argtypes = [C.c_uint32, C.POINTER(C.c_uint8), C.POINTER(C.c_float)]
    lib.zo_zone_planes.restype = C.c_int

    def get(gid):
        order, reach = (C.c_uint8 * 119)(), (C.c_float * 119)()
        count = lib.zo_zone_planes(gid, order, reach)
        return np.array(order[:count]), np.array(reach[:count], np.float64)

    assert lib.zo_zone_planes(11, (C.c_uint8 * 119)(), (C.c_float * 119)()) == -1
    return get


@pytest.mark.parametrize("group", GROUPS)
def test_reach_bounds_every_zone_point(zone_planes, ops64, ops32, group):
    gid = GROUPS.index(group)
    order, reach = zone_planes(gid)
    assert len(order) == 2 * len(ops64[group]) - 1
    assert sorted(order) == list(range(len(order)))          # a permutation of the planes
    assert np.all(np.diff(reach) >= 0)                       # sorted by reach
    for ops in (ops32[group], ops64[group]):
        h = planes_of(ops)
        x = qvm.normalize(qvm.fold(qvm.haar(200_000, 31 + gid), gid, ops, f32=False))
        dots = x @ h.T                                       # every zone point, every plane
        assert dots.min() >= -1e-9                           # the fold lands in the zone
        least = dots.min(axis=0)[order]
        assert np.all(least >= reach), (group, least[least < reach], reach[least < reach])
    if group in FACES:
        # The planes that touch the zone (its faces) come first with reach -1; every other
        # plane keeps a positive distance from the zone.
        touching = int((reach < 0).sum())
        assert touching == FACES[group]
        assert np.all(reach[touching:] > 0.1)
    else:
        assert np.all(reach == -1.0)  # cyclic groups: the zone has no vertices, every plane is tested
