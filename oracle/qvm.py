"""FP64 NumPy restatement of zxtalori's QVM repulsion path.  TEST INFRASTRUCTURE ONLY.

This module is the parity oracle: tests/ compare the CUDA engine against it, and it is
pinned against golden vectors produced by the reference's own dense models
(tests/golden/make_golden.py imports tests/test_pair_kernels.py:reference,
tests/test_measures.py:expected_measures and tests/test_near_field.py:near_reference).
The product never imports it.

Conventions follow the reference: quaternions are scalar first, symmetry acts on the
right (q*g), an orbit is {+-q_j g_k}. Citations are path:line in the reference project.
"""
from __future__ import annotations

import math

import numpy as np

GROUPS = ("C2", "C3", "C4", "C6", "D2", "D3", "D4", "D6", "T", "O", "I")
ORDER = {"C2": 2, "C3": 3, "C4": 4, "C6": 6, "D2": 4, "D3": 6, "D4": 8, "D6": 12, "T": 12, "O": 24, "I": 60}
PI = math.pi


# ---------------------------------------------------------------- quaternions
def qmul(a, b):
    """Hamilton product, scalar first (shaders/pairs.wgsl:22-24)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    w = a[..., 0] * b[..., 0] - (a[..., 1:] * b[..., 1:]).sum(-1)
    v = a[..., :1] * b[..., 1:] + b[..., :1] * a[..., 1:] + np.cross(a[..., 1:], b[..., 1:])
    return np.concatenate([w[..., None], v], axis=-1)


def normalize(a):
    a = np.asarray(a, np.float64)
    return a / np.linalg.norm(a, axis=-1, keepdims=True)


def operators(group, table):
    """Operator rows of `group` from a {name: (|K|,4)} table (src/groups.zig:24-201)."""
    return np.asarray(table[group], np.float64)


# ---------------------------------------------------------------- Haar sampler
def hash32(v):
    """Integer hash of shaders/haar.wgsl:3 (xorshift-multiply, two rounds), uint32 wraparound."""
    x = np.asarray(v, dtype=np.uint64) & 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return x.astype(np.uint32)


def _unit(v):
    """(f32(hash>>8)+0.5)/2^24, exact in float32 (shaders/haar.wgsl:4)."""
    return ((hash32(v) >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) / np.float32(16777216.0)


def haar(count, seed):
    """Shoemake uniform quaternions from the seeded hash (shaders/haar.wgsl:5-10).

    u, a, b are formed in float32 exactly as the shader forms them; the quaternion is
    evaluated in FP64 from those values and rounded once to float32 (the engine does the
    same on the GPU, so both agree to the last bit up to FP64 sin/cos ties).
    """
    i = np.arange(count, dtype=np.uint64)
    base = hash32(i ^ np.uint64(int(hash32(np.uint64(seed)))))
    two_pi = np.float32(6.28318530718)
    u = _unit(base.astype(np.uint64))
    a = two_pi * _unit(base.astype(np.uint64) + 1)
    b = two_pi * _unit(base.astype(np.uint64) + 2)
    u64, a64, b64 = u.astype(np.float64), a.astype(np.float64), b.astype(np.float64)
    su, sv = np.sqrt(u64), np.sqrt(1.0 - u64)
    q = np.stack([su * np.cos(b64), sv * np.sin(a64), sv * np.cos(a64), su * np.sin(b64)], axis=-1)
    return q.astype(np.float32)


# ---------------------------------------------------------------- fundamental-zone fold
_T6, _T8, _T12 = 0.5773502691896258, 0.4142135623730951, 0.2679491924311227
_C6, _S45 = 0.8660254037844386, 0.7071067811865476


def in_zone(p, gid, ops):
    """Homogeneous zone inequalities per group (shaders/state.wgsl:6-29), FP64 constants."""
    a = np.abs(p[..., 1:])
    w = p[..., 0]
    ax, ay, az = a[..., 0], a[..., 1], a[..., 2]
    if gid == 0:
        return az <= w
    if gid == 1:
        return az <= _T6 * w
    if gid == 2:
        return az <= _T8 * w
    if gid == 3:
        return az <= _T12 * w
    if gid == 4:
        return np.maximum(np.maximum(ax, ay), az) <= w
    if gid == 5:
        return (az <= _T6 * w) & (np.maximum(ax, 0.5 * ax + _C6 * ay) <= w)
    if gid == 6:
        return (az <= _T8 * w) & (np.maximum(np.maximum(ax, ay), _S45 * (ax + ay)) <= w)
    if gid == 7:
        m, n = np.maximum(ax, ay), np.minimum(ax, ay)
        return (az <= _T12 * w) & (np.maximum(m, _C6 * m + 0.5 * n) <= w)
    if gid == 8:
        return ax + ay + az <= w
    if gid == 9:
        return (np.maximum(np.maximum(ax, ay), az) <= _T8 * w) & (ax + ay + az <= w)
    # I: inner/outer shortcuts, then the twelve five-fold face rotations.
    inside = np.ones(p.shape[:-1], bool)
    for k in range(1, len(ops)):
        if abs(abs(ops[k, 0]) - 0.8090169943749475) < 1e-5:
            inside &= ~(np.abs((p * ops[k]).sum(-1)) > w)
    return np.where(w > 0.9510566, True, np.where(w < 0.9256147, False, inside))


def _flush(q32):
    """Exponent rescale of shaders/state.wgsl:31-40: components whose float32 exponent,
    rescaled so the largest is in [1,2), would be subnormal (or are zero/subnormal) become
    signed zeros; the rest keep their value (the power-of-two scale cancels in normalize)."""
    bits = np.ascontiguousarray(q32, np.float32).view(np.uint32)
    e = ((bits >> 23) & 255).astype(np.int64)
    emax = e.max(axis=-1, keepdims=True)
    keep = (e > 0) & (e + 127 - emax > 0)
    out = np.where(keep, q32.astype(np.float64), np.copysign(0.0, q32.astype(np.float64)))
    return out


def fold(q, gid, ops, f32=True):
    """Each quaternion to its zone representative (shaders/state.wgsl:30-46; engine.zig:233).

    Normalise (with the float32 rescale/flush when `f32`), take w >= 0, keep it if it is in
    the zone, else the image p*g_k with the largest |w| (first maximum wins), sign fixed and
    normalised. Arithmetic is FP64; with `f32` the input is float32 and the result is
    rounded to float32 (the engine's FP32 mode), else FP64 throughout (its FP64 mode).
    """
    q = np.asarray(q)
    p = _flush(q.astype(np.float32)) if f32 else np.asarray(q, np.float64).copy()
    p = normalize(p)
    p = np.where(p[..., :1] < 0, -p, p)
    inside = in_zone(p, gid, ops)
    best = p.copy()
    w = p[..., 0].copy()
    for k in range(len(ops)):
        c = qmul(p, ops[k])
        better = np.abs(c[..., 0]) > w
        c = np.where(c[..., :1] >= 0, c, -c)
        best = np.where(better[..., None], c, best)
        w = np.where(better, np.abs(c[..., 0]), w)
    out = np.where(inside[..., None], p, normalize(best))
    return out.astype(np.float32) if f32 else out


# ---------------------------------------------------------------- pair kernels
def mean_radius(count):
    """d_r: half the m solving pi(m - sin m) = pi^2/count by 60 bisections (src/pairs.zig:205-215)."""
    target = PI * PI / count
    lo, hi = 0.0, PI
    for _ in range(60):
        middle = 0.5 * (lo + hi)
        if PI * (middle - math.sin(middle)) < target:
            lo = middle
        else:
            hi = middle
    return 0.25 * (lo + hi)


def quey_pair(x, y, dm2, dp2):
    """One Quey pair (shaders/pairs.wgsl:250-262): returns force xyz, curvature, energy, angle.

    a = 2 atan(sqrt(near/far)) is the half-angle form of the S3 angle to the nearer of +-y.
    """
    near = np.maximum(np.minimum(dm2, dp2), 1e-30)
    far = np.maximum(np.maximum(dm2, dp2), 1e-30)
    t = np.sqrt(near / far)
    a = np.maximum(2.0 * np.arctan(t), 1e-12)
    b = PI - a
    a2, b2 = a * a + 1e-9, b * b + 1e-9
    a3, b3 = a * a * a + 1e-9, b * b * b + 1e-9
    sine = 2.0 * t / (1.0 + t * t) + 1e-9
    sign = np.where(dm2 <= dp2, 1.0, -1.0)
    direction = x[..., :1] * y[..., 1:] - y[..., :1] * x[..., 1:] + np.cross(x[..., 1:], y[..., 1:])
    along = sign * (b2 - a2) / (a2 * b2 * sine)
    force = -along[..., None] * direction
    curvature = (a3 + b3) / (a3 * b3)
    energy = PI / (a * b)
    return force, curvature, energy, a


def images(q, ops):
    """All images y = normalize(q_j g_k) (k=0: q_j itself), shape (|K|, N, 4), FP64."""
    q = np.asarray(q, np.float64)
    out = np.empty((len(ops),) + q.shape)
    for k, g in enumerate(ops):
        out[k] = q if k == 0 else normalize(qmul(q, g))
    return out


def _blocks(n, size):
    for start in range(0, n, size):
        yield start, min(n, start + size)


def _source_rows(n, sources):
    """The source indices that get rows: all of them, or the given subset (in its order)."""
    return np.arange(n) if sources is None else np.asarray(sources, np.int64)


def pair_rows(q, ops, full=False, block=256, sources=None):
    """Dense FP64 per-source rows over every image j*g_k (shaders/pairs.wgsl:151-244, 266-308).

    Returns a dict of per-source arrays:
      force (N,3), curvature, energy (Quey, own orbit excluded), nearest (min chord^2 over
      every image but the identity self pair) and nearest_source (its source index, first
      of equal chords in (k, j) order); with `full` also riesz1/2/3, green and log (all
      pairs but the identity self pair, plus the self pair's analytic antipode).
    With `sources`, only those sources get rows (the arrays follow its order), still
    summed over every image of the whole sample.
    """
    x_all = normalize(q)
    n = len(x_all)
    src = _source_rows(n, sources)
    m = len(src)
    ys = images(x_all, ops)
    res = {"force": np.zeros((m, 3)), "curvature": np.zeros(m), "energy": np.zeros(m),
           "nearest": np.full(m, 4.0), "nearest_source": np.full(m, -1, np.int64)}
    if full:
        for key in ("riesz1", "riesz2", "riesz3", "green", "log"):
            res[key] = np.zeros(m)
    for i0, i1 in _blocks(m, block):
        rows = src[i0:i1]
        x = x_all[rows][:, None, :]
        for k in range(len(ops)):
            y = ys[k][None, :, :]
            minus, plus = x - y, x + y
            dm2 = (minus * minus).sum(-1)
            dp2 = (plus * plus).sum(-1)
            own = rows[:, None] == np.arange(n)[None, :]
            self_pair = own if k == 0 else np.zeros_like(own)
            chord = np.where(self_pair, 4.0, np.minimum(dm2, dp2))
            j = chord.argmin(-1)
            c = chord[np.arange(len(rows)), j]
            better = c < res["nearest"][i0:i1]
            res["nearest"][i0:i1] = np.where(better, c, res["nearest"][i0:i1])
            res["nearest_source"][i0:i1] = np.where(better, j, res["nearest_source"][i0:i1])
            force, curv, energy, angle = quey_pair(x, y, dm2, dp2)
            keep = ~own
            res["force"][i0:i1] += np.where(keep[..., None], force, 0).sum(1)
            res["curvature"][i0:i1] += np.where(keep, curv, 0).sum(1)
            res["energy"][i0:i1] += np.where(keep, energy, 0).sum(1)
            if full:
                keep = ~self_pair
                im = 1.0 / np.sqrt(np.maximum(dm2, 1e-30))
                ip = 1.0 / np.sqrt(np.maximum(dp2, 1e-30))
                res["riesz1"][i0:i1] += np.where(keep, im + ip, 0).sum(1)
                res["riesz2"][i0:i1] += np.where(keep, im * im + ip * ip, 0).sum(1)
                res["riesz3"][i0:i1] += np.where(keep, im ** 3 + ip ** 3, 0).sum(1)
                cot = np.abs(dp2 - dm2) * 0.5 * im * ip
                green = ((PI - 2.0 * angle) * cot - 1.0) / (4.0 * PI * PI)
                res["green"][i0:i1] += np.where(keep, green, 0).sum(1)
                with np.errstate(divide="ignore"):
                    lg = -0.5 * np.log(np.where(keep, dm2 * dp2, 1.0)) + 0.5
                res["log"][i0:i1] += np.where(keep, lg, 0).sum(1)
    if full:
        res["riesz1"] += 0.5
        res["riesz2"] += 0.25
        res["riesz3"] += 0.125
        res["green"] += -3.0 / (8.0 * PI * PI)
        res["log"] += -math.log(2.0) + 0.25
    return res


def near_radius(n, order, delta):
    """Cutoff angle r = min(1.5, delta d_r) on S3 and its squared chord (src/near.zig:95, 176)."""
    r = min(1.5, delta * mean_radius(n * order))
    return r, (2.0 * math.sin(r / 2.0)) ** 2


def near_pair(x, y, dm2, dp2, r, taper=0.5):
    """Windowed Quey pair (shaders/pairs.wgsl:352-361): C1 window 1 - s^2(3-2s) from taper*r to r."""
    force, curv, energy, a = quey_pair(x, y, dm2, dp2)
    width = 1.0 / max(1e-9, (1.0 - taper) * r)
    s = np.clip((a - taper * r) * width, 0.0, 1.0)
    window = 1.0 - s * s * (3.0 - 2.0 * s)
    slope = -6.0 * s * (1.0 - s) * width
    sign = np.where(dm2 <= dp2, 1.0, -1.0)
    direction = x[..., :1] * y[..., 1:] - y[..., :1] * x[..., 1:] + np.cross(x[..., 1:], y[..., 1:])
    extra = sign * energy * slope / np.maximum(np.sin(a), 1e-9)
    active = s > 0
    force = np.where(active[..., None], window[..., None] * force + extra[..., None] * direction, force)
    curv = np.where(active, window * curv, curv)
    energy = np.where(active, window * energy, energy)
    return force, curv, energy


def near_rows(q, ops, delta, taper=0.5, block=256, sources=None):
    """Dense FP64 near-field rows (shaders/pairs.wgsl:363-416 semantics, src/near.zig:1-11).

    Source i feels every orbit point (either sign of every image) whose chord to it is at
    most 2 sin(r/2), its own orbit excluded; the nearest is over those points and its own
    images other than the identity one (within the cutoff, as the kernel sees them).
    Every image is tested (no shell, no grid), so this pins any faster membership rule.
    With `sources`, only those sources get rows (the arrays follow its order).
    """
    x_all = normalize(q)
    n = len(x_all)
    src = _source_rows(n, sources)
    m = len(src)
    order = len(ops)
    r, cut = near_radius(n, order, delta)
    flat = images(x_all, ops).reshape(-1, 4)  # image k*n + j
    res = {"force": np.zeros((m, 3)), "curvature": np.zeros(m), "energy": np.zeros(m),
           "nearest": np.full(m, 4.0), "nearest_source": np.full(m, -1, np.int64), "radius": r, "cut": cut}
    # Candidates first: for unit vectors |x - s y|^2 = 2 - 2 s x.y, which a matrix product
    # gives for every image at once; a slack of 1e-12 keeps every point within the cutoff.
    # Membership itself is then decided on the difference form, as the kernel's semantics
    # state it, and only the members' pair terms are evaluated.
    for i0, i1 in _blocks(m, block):
        rows = src[i0:i1]
        x = x_all[rows]
        dot = x @ flat.T
        for sgn, sign in enumerate((1.0, -1.0)):
            bi, fi = np.nonzero(2.0 - 2.0 * sign * dot <= cut + 1e-12)
            if len(bi) == 0:
                continue
            xs, y = x[bi], sign * flat[fi]
            minus, plus = xs - y, xs + y
            dm2 = (minus * minus).sum(-1)
            dp2 = (plus * plus).sum(-1)
            k, j = fi // n, fi % n
            inside = dm2 <= cut
            own = rows[bi] == j
            identity = own & (k == 0) & (sign > 0)
            # Nearest: smallest chord, first in (k, sign, j) order among equal ones.
            cand = inside & ~identity
            if cand.any():
                b, c, kk, jj = bi[cand], dm2[cand], k[cand], j[cand]
                pick_order = np.lexsort((jj, kk, c, b))  # by row, chord, then operator, then source
                first = np.ones(len(pick_order), bool)
                first[1:] = b[pick_order][1:] != b[pick_order][:-1]
                win = pick_order[first]
                rb, rc, rk, rj = b[win] + i0, c[win], kk[win], jj[win]
                held_k = res.setdefault("_k", np.full(m, 1 << 30))
                held_s = res.setdefault("_s", np.full(m, 2))
                cur = res["nearest"][rb]
                better = (rc < cur) | ((rc == cur) & ((rk < held_k[rb]) | ((rk == held_k[rb]) & (sgn < held_s[rb]))))
                res["nearest"][rb[better]] = rc[better]
                res["nearest_source"][rb[better]] = rj[better]
                held_k[rb[better]] = rk[better]
                held_s[rb[better]] = sgn
            pick = inside & ~own
            if not pick.any():
                continue
            xp, yp = xs[pick][:, None, :], y[pick][:, None, :]
            force, curv, energy = near_pair(xp, yp, dm2[pick][:, None], dp2[pick][:, None], r, taper)
            b = bi[pick]
            for a in range(3):
                res["force"][i0:i1, a] += np.bincount(b, force[:, 0, a], minlength=i1 - i0)
            res["curvature"][i0:i1] += np.bincount(b, curv[:, 0], minlength=i1 - i0)
            res["energy"][i0:i1] += np.bincount(b, energy[:, 0], minlength=i1 - i0)
    res.pop("_k", None)
    res.pop("_s", None)
    return res


# ---------------------------------------------------------------- measures
C_GREEN = 3 ** (5 / 3) / (5 * (2 * PI * PI) ** (1 / 3) * (4 * PI) ** (2 / 3))


def separation_deg(nearest_chord2):
    """SO(3) angle of a squared S3 chord: 4 asin(min(1, sqrt(c)/2)) in degrees (src/pairs.zig:170)."""
    return 4.0 * math.degrees(math.asin(min(1.0, math.sqrt(max(nearest_chord2, 0.0)) / 2.0)))


def quick_measures(rows, order):
    """Quey energy, separation and force RMS of a force pass (src/pairs.zig:130-140, 182-199)."""
    n = len(rows["energy"])
    near = float(rows["nearest"].min())
    if near <= 0:
        raise ValueError("DuplicateOrientations")
    return {"quey_energy": float(rows["energy"].sum()) / (n * order * max(n - 1, 1)),
            "separation_deg": separation_deg(near),
            "force_rms": float(np.sqrt((rows["force"] ** 2).sum() / n))}


def full_measures(rows, order):
    """Energy ratios from full rows (src/pairs.zig:142-173)."""
    n = len(rows["energy"])
    out = quick_measures(rows, order)
    ext = 2.0 * order
    total = n * ext
    s = [ext * float(rows[k].sum()) for k in ("riesz1", "riesz2", "riesz3", "log", "green")]
    delta = (s[3] + 0.25 * total + math.log(total) * total / 3.0) / total
    out.update({
        "count_extended": total,
        "riesz_1": s[0] / (total * total * (8.0 / (3.0 * PI))),
        "riesz_2": s[1] / (total * total),
        "riesz_3": s[2] / ((2.0 / (3.0 * PI)) * total * total * math.log(total)),
        "green_ratio": s[4] / (-C_GREEN * total ** (4.0 / 3.0)),
        "log_ratio": delta / (-5.0 / 12.0),
    })
    return out


def ratio_limit(order):
    """Largest N whose energy ratios measure() computes: floor(sqrt(5e10/|K|)) (src/engine.zig:348-351)."""
    return int(math.floor(math.sqrt(5e10 / order)))


# ---------------------------------------------------------------- BB relaxation
def exact_median(values):
    """Mean of the lower and upper middle values of max(c, 0), at least 1e-12 (shaders/relax.wgsl:76-134)."""
    v = np.sort(np.where(values > 0, values, 0.0))
    n = len(v)
    return max(1e-12, 0.5 * (v[(n - 1) // 2] + v[n // 2]))


class Relax:
    """Barzilai-Borwein relaxation with the reference's step rules (shaders/relax.wgsl,
    src/pairs.zig:339-413, src/engine.zig:896-937), FP64 throughout.

    State persists across calls like RelaxState: the iteration counter, the previous force
    and move per source. `f32` rounds positions to float32 after every fold (the engine's
    FP32 storage); otherwise positions stay FP64.
    """

    def __init__(self, q, gid, ops, delta=0.0, f32=False, fixed=None, rows_fn=None):
        self.q = np.asarray(q, np.float32 if f32 else np.float64).copy()
        self.gid, self.ops, self.delta, self.f32 = gid, ops, float(delta), f32
        self.fixed = fixed
        self.iteration = 0
        n = len(self.q)
        self.prev_force = np.zeros((n, 3))
        self.prev_move = np.zeros((n, 3))
        self.rows_fn = rows_fn
        self.history = []

    def rows(self, q):
        if self.rows_fn is not None:
            return self.rows_fn(q)
        if self.delta > 0:
            return near_rows(q, self.ops, self.delta)
        return pair_rows(q, self.ops)

    def step(self, rows=None, step_scale=1.0):
        q = self.q.astype(np.float64)
        n = len(q)
        order = len(self.ops)
        rows = self.rows(q) if rows is None else rows
        radius = mean_radius(n * order)
        alpha0 = (0.8 / 3.4) * radius ** 3
        f = rows["force"]
        flags = 0
        if not np.isfinite(f).all():
            flags |= 1
        if not (rows["nearest"] > 0).all():
            flags |= 2
        mask = np.ones(n, bool)
        if self.fixed is not None:
            mask[self.fixed] = False
        first = self.iteration == 0
        if not first:
            s = self.prev_move[mask]
            yv = f[mask] - self.prev_force[mask]
            sty, yty, sts = float((s * yv).sum()), float((yv * yv).sum()), float((s * s).sum())
        ftf = float((f * f).sum())
        energy = float(rows["energy"].sum())
        median = exact_median(rows["curvature"])
        alpha = alpha0
        if not first:
            a1 = abs(sty / yty) if abs(yty) > 1e-20 else alpha0
            a2 = abs(sts / sty) if abs(sty) > 1e-20 else alpha0
            alpha = min(max(a1 if self.iteration % 2 == 1 else a2, 1e-12), max(1.0, 10.0 * radius))
        self.iteration += 1
        record = {"alpha": alpha, "median": median, "flags": flags, "ftf": ftf, "energy": energy}
        if flags:
            self.history.append(record)
            return record
        scale = alpha * step_scale / np.maximum(1e-6, rows["curvature"] / median + 1e-2)
        size = np.linalg.norm(f, axis=-1) * scale
        clip = np.minimum(1.0, 0.5 * radius / np.maximum(size, 1e-12))
        d = f * (scale * clip)[:, None]
        self.prev_force = f.copy()
        self.prev_move = d.copy()
        angle = np.linalg.norm(d, axis=-1)
        sinc = np.where(angle > 1e-4, np.sin(angle) / np.where(angle > 0, angle, 1.0), 1.0 - angle * angle / 6.0)
        rot = np.concatenate([np.cos(angle)[:, None], d * sinc[:, None]], axis=-1)
        moved = normalize(qmul(rot, q))
        moved = np.where(moved[:, :1] < 0, -moved, moved)
        record["step"] = float((size * clip)[mask].max()) if mask.any() else 0.0
        if self.fixed is not None:
            moved[self.fixed] = (1.0, 0.0, 0.0, 0.0)
            self.prev_force[self.fixed] = 0
            self.prev_move[self.fixed] = 0
        # Move and fold are one FP64 pass (the engine fuses them); FP32 storage rounds once.
        folded = fold(moved, self.gid, self.ops, f32=False)
        self.q = folded.astype(np.float32) if self.f32 else folded
        self.history.append(record)
        return record

    def run(self, steps):
        for _ in range(steps):
            self.step()
        return self.q


def nearest_degrees(rows):
    """Per-source nearest orbit neighbour as an SO(3) angle in degrees (shaders/pairs.wgsl:428-434)."""
    c = np.sqrt(np.maximum(rows["nearest"], 0.0)) * 0.5
    return np.degrees(4.0 * np.arcsin(np.minimum(1.0, c)))
