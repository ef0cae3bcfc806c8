"""The epilogue's first Johnson-Cook screen calls no particle elastic that the
FP32 screen would not.

jc_clearly_elastic (iwf_mfree_gpu_3d_b200/csrc/mfree_device.cuh) bounds the
yield stress from below by A (1 - 1.001 theta^m), with theta^m from the
approximate exp2/log2 instructions, and takes a particle as elastic when its
von Mises stress is under 0.98 of that bound.  The step then gives the same
bits as with the FP32 screen alone (elastic under 0.99 of
jc_yield_stress_screen) only if 0.98 of the bound never exceeds 0.99 of the
screen.  This checks that on seeded samples, each side at the far end of its
error: the bound with theta^m under-estimated by the approximate instructions'
error (2^-21 relative on the exponential, 2^-21 on the logarithm scaled by
|log2 theta| and m), the screen with every powf/logf result moved 4 ulp and
every product 1 ulp towards a smaller yield stress.  The samples cover the
benchmark material (the steel of the cutting scenes) and wide parameter
ranges, up to the bound's own limit 1 - theta^m >= 1e-3.
"""
import numpy as np

from iwf_mfree_gpu_3d_b200 import scenes

ULP = 2.0 ** -23


def screen_low(A, B, C, n, m, eps, epsd, theta, eref):
    """jc_yield_stress_screen with every rounding taken towards a smaller
    yield stress (relative errors as bounds, in float64)."""
    pw = np.power(eps, n) * (1 - 4 * ULP)
    a = (A + B * pw) * (1 - ULP)
    ed = epsd / eref
    b = np.where(ed > 1.0, 1.0 + C * np.log(np.maximum(ed, 1.0)) * (1 - 4 * ULP),
                 np.power(1.0 + ed, C) * (1 - 4 * ULP))
    c = (1.0 - np.power(theta, m) * (1 + 4 * ULP)) * (1 - ULP)
    return a * b * (1 - ULP) * c * (1 - ULP)


def bound_high(A, m, theta):
    """The first screen's bound A (1 - 1.001 p) with p = theta^m as small as
    the approximate instructions can make it, and its flag c >= 1e-3."""
    l2 = np.log2(np.maximum(theta, 1e-300))
    err = 2.0 ** -21 * (1.0 + m * np.maximum(1.0, np.abs(l2)))
    p = np.power(theta, m) * np.exp2(-err) * (1 - 2.0 ** -21)
    c = 1.0 - 1.001 * p
    return A * c * (1 + 2 * ULP), c >= 1e-3


def check(A, B, C, n, m, eps, epsd, theta, eref):
    lo = screen_low(A, B, C, n, m, eps, epsd, theta, eref)
    hi, ok = bound_high(A, m, theta)
    bad = ok & (0.98 * hi > 0.99 * lo)
    assert not bad.any(), (np.flatnonzero(bad)[:5], hi[bad][:5], lo[bad][:5])
    return int(ok.sum())


def test_benchmark_material():
    jc = scenes.STEEL_JC
    rng = np.random.default_rng(7)
    k = 200_000
    eps = np.concatenate([np.zeros(1000), rng.uniform(0, 2, k), 10.0 ** rng.uniform(-12, 0, k)])
    epsd = np.concatenate([np.zeros(1000), 10.0 ** rng.uniform(-12, 3, k), rng.uniform(0, 1e-5, k)])
    theta = np.concatenate([np.zeros(1000), rng.uniform(0, 1, k), 1 - 10.0 ** rng.uniform(-4, 0, k)])
    n = check(jc["A"], jc["B"], jc["C"], jc["n"], jc["m"], eps, epsd, theta, jc["eps_dot_ref"])
    assert n > k  # most samples are within the bound's range


def test_wide_parameter_ranges():
    rng = np.random.default_rng(11)
    k = 400_000
    A = 10.0 ** rng.uniform(-6, 3, k)
    B = np.where(rng.random(k) < 0.1, 0.0, 10.0 ** rng.uniform(-6, 3, k))
    C = np.where(rng.random(k) < 0.1, 0.0, rng.uniform(0, 0.5, k))
    n = rng.uniform(0.01, 2.0, k)
    m = 10.0 ** rng.uniform(-1, 1, k)
    eps = np.where(rng.random(k) < 0.2, 0.0, 10.0 ** rng.uniform(-10, 1, k))
    epsd = np.where(rng.random(k) < 0.2, 0.0, 10.0 ** rng.uniform(-10, 4, k))
    theta = np.where(rng.random(k) < 0.1, 0.0, rng.uniform(0, 1, k))
    eref = 10.0 ** rng.uniform(-8, 0, k)
    assert check(A, B, C, n, m, eps, epsd, theta, eref) > k // 2
