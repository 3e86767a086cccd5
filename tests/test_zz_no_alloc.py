"""zo_pair_rows_noalloc: the all-pairs force pass for callers that cannot allocate device
memory (their buffers come from a framework's own pool or a fixed reservation, or their
thread must not risk an allocation). The entry point takes the caller's device buffers and
uses only a fixed scratch array inside the library.

Checked through the C ABI against the engine's own force pass (zo_debug_rows) on the same
float32 positions, on two calls in a row: the second runs on the scratch the first left
behind. Same kernel, so the tolerance is the FP64 summation-order one: 1e-12 relative.
Collected last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bind(engine):
    lib = engine.api._library()
    fn = lib.zo_pair_rows_noalloc
    fn.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    fn.restype = C.c_int
    return fn


def run(fn, group_id, q_dev, n, out_dev):
    err = C.create_string_buffer(256)
    rc = fn(group_id, q_dev.data_ptr(), n, out_dev.data_ptr(), None, err, 256)
    return rc, err.value.decode()


@pytest.mark.parametrize("group,count", [("O", 1000), ("I", 300), ("C2", 5000), ("D6", 40000)])
def test_no_alloc_matches_engine_force_pass(engine, group, count):
    import torch

    fn = bind(engine)
    with engine.haar(group, count, 23) as grid:
        q = grid.quaternions
        expected = grid.debug_rows(0)
    q_dev = torch.from_numpy(q).cuda()
    results = []
    for _ in range(2):
        out = torch.full((6 * count,), float("nan"), dtype=torch.float64, device="cuda")
        rc, msg = run(fn, engine.GROUPS.index(group), q_dev, count, out)
        assert rc == 0, msg
        torch.cuda.synchronize()
        results.append(out.cpu().numpy())
    for got in results:
        force = got[:4 * count].reshape(count, 4)
        np.testing.assert_allclose(force[:, :3], expected[:, :3], rtol=1e-12,
                                   atol=1e-12 * np.abs(expected[:, :3]).max())
        np.testing.assert_allclose(force[:, 3], expected[:, 3], rtol=1e-12)
        np.testing.assert_allclose(got[4 * count:5 * count], expected[:, 4], rtol=1e-12)
        np.testing.assert_array_equal(got[5 * count:], expected[:, 5])
    np.testing.assert_array_equal(results[0], results[1])


def test_no_alloc_rejects_sizes_beyond_its_scratch(engine):
    import torch

    fn = bind(engine)
    q_dev = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    out = torch.zeros((24,), dtype=torch.float64, device="cuda")
    rc, msg = run(fn, 9, q_dev, 65537, out)
    assert rc == -2 and "65536" in msg
    rc, msg = run(fn, 11, q_dev, 4, out)
    assert rc == -1 and "group" in msg


def test_no_alloc_rows_do_not_depend_on_representative_signs(engine):
    """Antipodal invariance of the all-pairs kernel on unfolded input (this entry point takes
    positions as given, with no zone fold): negating every other quaternion leaves force,
    curvature, energy and nearest chord unchanged (tests/test_pair_kernels.py:131-135); each
    pair picks its near twin by the sign of x.y either way, so only rounding may differ."""
    import torch

    fn = bind(engine)
    with engine.haar("D3", 2000, 5) as grid:
        q = grid.quaternions
    signed = q.copy()
    signed[::2] *= -1
    rows = []
    for values in (q, signed):
        out = torch.zeros((6 * len(q),), dtype=torch.float64, device="cuda")
        rc, msg = run(fn, engine.GROUPS.index("D3"), torch.from_numpy(values).cuda(), len(q), out)
        assert rc == 0, msg
        torch.cuda.synchronize()
        rows.append(out.cpu().numpy())
    n = len(q)
    a, b = rows
    fa, fb = a[:4 * n].reshape(n, 4), b[:4 * n].reshape(n, 4)
    # The left-tangent force vec(y x*) is unchanged by x -> -x (the near twin flips with it).
    assert np.abs(fa[:, :3] - fb[:, :3]).max() < 1e-5 * np.abs(fa[:, :3]).max()
    np.testing.assert_allclose(fa[:, 3], fb[:, 3], rtol=1e-5)
    np.testing.assert_allclose(a[4 * n:5 * n], b[4 * n:5 * n], rtol=1e-5)
    np.testing.assert_allclose(a[5 * n:], b[5 * n:], rtol=1e-5)
