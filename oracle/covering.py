"""FP64 covering-radius oracle (Qhull).  TEST INFRASTRUCTURE ONLY.

The spherical Delaunay triangulation of a sample's full orbit {+-q_j g_k} on S3 is its
convex hull in R4: every hull facet's cap (the points of S3 beyond the facet's hyperplane)
is empty, and the covering radius is the angular radius of the largest such cap. This is
the reference's own test oracle, restated: tests/test_covering.py:8-15 (full_orbit_covering)
and tests/test_point_values.py:15-20, 28-37 (per-point largest cap and Voronoi faces). The
simplex bound is the series of src/covering_reference.zig:4-15. The product never imports
this module.
"""
from __future__ import annotations

import math

import numpy as np

# src/covering_reference.zig:7 (coefficients of the simplex-bound series in t^2, t = count^-1/3).
SIMPLEX_SERIES = (1.889832101454757, 0.573930763512449, 0.581069217539205, 0.859789414116394,
                  1.490131881944242, 2.791922498626376, 5.481645765756282, 11.12163594341394)


def _qmul(a, b):
    w = a[..., :1] * b[..., :1] - (a[..., 1:] * b[..., 1:]).sum(-1, keepdims=True)
    v = a[..., :1] * b[..., 1:] + b[..., :1] * a[..., 1:] + np.cross(a[..., 1:], b[..., 1:])
    return np.concatenate([w, v], axis=-1)


def orbit(q, ops):
    """The full orbit, images first then their antipodes, and each point's source index
    (tests/test_point_values.py:15-20): point k*n + j is q_j g_k (unit), 2|K|n points."""
    q = np.asarray(q, np.float64)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    ops = np.asarray(ops, np.float64)
    ops = ops / np.linalg.norm(ops, axis=1, keepdims=True)
    images = np.concatenate([_qmul(q, np.broadcast_to(op, q.shape)) for op in ops])
    images /= np.linalg.norm(images, axis=1, keepdims=True)
    return np.concatenate([images, -images]), np.tile(np.arange(len(q)), 2 * len(ops))


def simplex_degrees(count):
    """Simplex bound on the covering radius of `count` points (images and antipodes
    included), SO(3) degrees (src/covering_reference.zig:4-15)."""
    if count <= 0:
        return None
    t = (1.0 / count) ** (1.0 / 3.0)
    value = 0.0
    for c in reversed(SIMPLEX_SERIES):
        value = c + t * t * value
    return t * value * 360.0 / math.pi


def covering(q, ops):
    """Covering radius (SO(3) degrees) of the sample, each point's largest incident cap
    (degrees) and Voronoi face count, and the centre of the largest cap (a unit quaternion).

    Radius: 2 acos(min facet offset) (tests/test_covering.py:15). Per point: the largest cap
    of any facet touching an image of the point, and the number of distinct hull vertices
    sharing a facet with its identity image (tests/test_point_values.py:28-37).
    """
    from scipy.spatial import ConvexHull

    points, source = orbit(q, ops)
    n = len(q)
    hull = ConvexHull(points)
    normals = hull.equations[:, :4]
    offsets = -hull.equations[:, 4] / np.linalg.norm(normals, axis=1)
    radii = np.degrees(2 * np.arccos(np.clip(offsets, -1, 1)))
    largest = np.zeros(n)
    neighbours = [set() for _ in range(n)]
    for facet, radius in zip(hull.simplices, radii):
        for v in facet:
            if v < n:
                neighbours[v].update(int(w) for w in facet if w != v)
            largest[source[v]] = max(largest[source[v]], radius)
    top = int(np.argmax(radii))
    witness = normals[top] / np.linalg.norm(normals[top])
    return {"radius_deg": float(radii.max()), "point_covering": largest,
            "faces": np.array([len(s) for s in neighbours]), "witness": witness,
            "facets": len(hull.simplices)}
