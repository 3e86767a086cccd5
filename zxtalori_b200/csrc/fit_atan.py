"""Fit the float32 arctangent used by the pair kernels, and the short-chord forms.

atan(t) = t * P(t^2) on t in [0, 1] (the half-angle ratio chord(near)/chord(far) never
exceeds 1). P is a degree-8 polynomial in s = t^2 whose coefficients minimise the
maximum relative error (iteratively reweighted least squares on Chebyshev nodes,
converging to the equioscillating minimax fit). The kernels evaluate 2*atan(t) with
the coefficients doubled (an exact scaling).

For near-field cutoffs up to 0.4 rad the gather works from the squared chord d <= 0.25
alone: the angle 2 asin(sqrt(d)/2) = sqrt(d) (1 + d Pa(d)) and its sine
sqrt(d) sqrt(1 - d/4) = sqrt(d) (1 + d Ps(d)), Pa and Ps quadratics fitted the same way
(relative error of 1 + d P). Run to reproduce the tables in qvm_device.cuh:
python zxtalori_b200/csrc/fit_atan.py
"""
import numpy as np


def fit(degree=8, iterations=60, t_max=1.0):
    s = (np.cos(np.linspace(0, np.pi, 4000)) * 0.5 + 0.5) * t_max * t_max

    def target(v):
        t = np.sqrt(v)
        return np.where(v > 0, np.arctan(t) / np.where(t > 0, t, 1), 1.0)

    w = np.ones_like(s)
    c = None
    for _ in range(iterations):
        scale = w / target(s)
        a = np.vander(s, degree + 1, increasing=True) * scale[:, None]
        c, *_ = np.linalg.lstsq(a, target(s) * scale, rcond=None)
        err = np.vander(s, degree + 1, increasing=True) @ c / target(s) - 1
        w = w * (1 + 4 * np.abs(err) / np.abs(err).max())
    grid = np.linspace(0, t_max * t_max, 2_000_001)
    worst = np.abs(np.polyval(c[::-1], grid) / target(grid) - 1).max()
    return c, worst


def fit_chord(target, degree=3, iterations=60, d_max=0.25):
    """1 + d P(d) ~ target(d) on [0, d_max], P of degree - 1, minimax in relative error."""
    d = (np.cos(np.linspace(0, np.pi, 4000)) * 0.5 + 0.5) * d_max
    d = d[d > 0]
    y = target(d)
    a0 = np.vander(d, degree, increasing=True) * d[:, None]
    w = np.ones_like(d)
    c = None
    for _ in range(iterations):
        scale = w / y
        c, *_ = np.linalg.lstsq(a0 * scale[:, None], (y - 1) * scale, rcond=None)
        err = (1 + a0 @ c) / y - 1
        w = w * (1 + 4 * np.abs(err) / np.abs(err).max())
    grid = np.linspace(d_max * 1e-9, d_max, 2_000_001)
    c32 = np.array([np.float32(v) for v in c], np.float64)
    worst = np.abs((1 + grid * np.polyval(c32[::-1], grid)) / target(grid) - 1).max()
    return c, worst


def chord_angle(d):
    return 2 * np.arcsin(np.sqrt(d) / 2) / np.sqrt(d)


def chord_sine(d):
    return np.sqrt(1 - d / 4)


if __name__ == "__main__":
    # The full range (any cutoff) and the short range used when the near-field cutoff
    # r <= 0.4 rad keeps t = tan(a/2) <= tan(0.2) < 0.21.
    for degree, t_max in ((8, 1.0), (3, 0.21)):
        coeffs, worst = fit(degree, t_max=t_max)
        print(f"t in [0, {t_max}], degree {degree} in t^2: max relative error {worst:.3e}")
        for k, v in enumerate(coeffs):
            print(f"  c{k} = {float(np.float32(2 * v)).hex()}f  // 2 * {v:+.10e}")
    for name, target in (("angle / sqrt(d)", chord_angle), ("sine / sqrt(d)", chord_sine)):
        coeffs, worst = fit_chord(target)
        print(f"{name} = 1 + d P(d), d in [0, 0.25], P quadratic: max relative error {worst:.3e}")
        for k, v in enumerate(coeffs):
            print(f"  p{k} = {float(np.float32(v)).hex()}f")
