"""Fit the float32 arctangent used by the pair kernels.

atan(t) = t * P(t^2) on t in [0, 1] (the half-angle ratio chord(near)/chord(far) never
exceeds 1). P is a degree-8 polynomial in s = t^2 whose coefficients minimise the
maximum relative error (iteratively reweighted least squares on Chebyshev nodes,
converging to the equioscillating minimax fit). The kernels evaluate 2*atan(t) with
the coefficients doubled (an exact scaling). Run to reproduce the table in
qvm_device.cuh:  python zxtalori_b200/csrc/fit_atan.py
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


if __name__ == "__main__":
    # The full range (any cutoff) and the short range used when the near-field cutoff
    # r <= 0.4 rad keeps t = tan(a/2) <= tan(0.2) < 0.21.
    for degree, t_max in ((8, 1.0), (3, 0.21)):
        coeffs, worst = fit(degree, t_max=t_max)
        print(f"t in [0, {t_max}], degree {degree} in t^2: max relative error {worst:.3e}")
        for k, v in enumerate(coeffs):
            print(f"  c{k} = {float(np.float32(2 * v)).hex()}f  // 2 * {v:+.10e}")
