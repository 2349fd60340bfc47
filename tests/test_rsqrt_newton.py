"""The split-precision metric's 1/sqrt(rho2) (rho2 = 1 + tan^2 x + tan^2 y in
[1, 3)): an FP32 approximation with relative error below 2^-22 (the bound of
the hardware's rsqrt.approx.f32) refined by one Newton-Raphson step
y' = y + y (1 - rho2 y^2) / 2, evaluated in FP64 as the stage kernel does.
One step squares the relative error (e' = 1.5 e^2 + e^3 / 2), so the result is
within 1.5e-13 of 1/sqrt(rho2) for every seed inside that bound (here also
rounded to FP32 once more, which the hardware's own result already is)."""
import numpy as np


def newton_rsqrt(rho2, seed):
    y0 = seed.astype(np.float64)
    e = 1.0 - rho2 * y0 * y0
    return 0.5 * y0 * e + y0


def test_one_newton_step_from_a_2pow22_seed():
    rho2 = np.linspace(1.0, 3.0, 200001)[:-1]
    exact = 1.0 / np.sqrt(rho2)
    for tilt in (-1.0, -0.5, 0.0, 0.5, 1.0):
        # the worst seeds the hardware bound allows, rounded to FP32
        seed = (exact * (1.0 + tilt * 2.0 ** -22)).astype(np.float32)
        rel = np.abs(newton_rsqrt(rho2, seed) - exact) / exact
        assert rel.max() < 1.5e-13, (tilt, rel.max())
