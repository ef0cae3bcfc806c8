"""The oracle against the reference's own functions (golden vectors).

tests/golden/ref_kat.npz holds outputs of the reference's cubic_spline,
lapl_pse, solve_eigen, sigma_yield and solve_secant compiled unchanged for the
host (tests/golden/make_golden.py).  The oracle's FP32 instantiation must
reproduce the kernel function bit for bit; the eigen solver and the PSE weight
differ only by the host's double-precision libm against float math (the
reference's host build resolves sqrt/acos/cos(float) to the double versions).
"""
import ctypes as C
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_kat.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_cubic_spline_bit_exact_fp32(oracle_lib, gold):
    L = oracle_lib.lib()
    pi, pj, hs, w = gold["spline_pi"], gold["spline_pj"], gold["spline_h"], gold["spline_w"]
    out = np.zeros(4)
    got = np.zeros_like(w)
    for k in range(len(pi)):
        L.orc_cubic_spline(32, _dp(pi[k].astype(np.float64)), _dp(pj[k].astype(np.float64)), float(hs[k]), _dp(out))
        got[k] = out
    np.testing.assert_array_equal(got.astype(np.float32), w)


def test_cubic_spline_fp64_close(oracle_lib, gold):
    L = oracle_lib.lib()
    pi, pj, hs, w = gold["spline_pi"], gold["spline_pj"], gold["spline_h"], gold["spline_w"]
    out = np.zeros(4)
    for k in range(0, len(pi), 3):
        L.orc_cubic_spline(64, _dp(pi[k].astype(np.float64)), _dp(pj[k].astype(np.float64)), float(hs[k]), _dp(out))
        scale = np.abs(w[k]).max() + 1e-30
        # FP64 against the FP32 reference: x_i - x_j of close float pairs loses bits
        assert np.abs(out - w[k]).max() / scale < 5e-5


def test_support_edges_in_golden(gold):
    # the fixture covers coincident particles, the support edge and outside
    w = gold["spline_w"]
    assert (w[:50] == 0).all()
    assert (w[:, 0] == 0).sum() > 500 and (w[:, 0] > 0).sum() > 1000


def test_pse_weight(oracle_lib, gold):
    L = oracle_lib.lib()
    pi, pj, hs, pse = gold["spline_pi"], gold["spline_pj"], gold["spline_h"], gold["pse"]
    got = np.array([L.orc_lapl_pse(32, _dp(pi[k].astype(np.float64)), _dp(pj[k].astype(np.float64)), float(hs[k]))
                    for k in range(len(pi))])
    np.testing.assert_allclose(got.astype(np.float32), pse, rtol=2e-6, atol=0)


def test_eigen_solver(oracle_lib, gold):
    L = oracle_lib.lib()
    A, ref = gold["eig_in"], gold["eig_out"]
    out = np.zeros(12)
    # FP64 restatement against the FP32 reference: near-repeated eigenvalues amplify float rounding
    for prec, tol in ((32, 2e-5), (64, 1e-4)):
        worst = 0.0
        for k in range(len(A)):
            L.orc_solve_eigen(prec, _dp(A[k].astype(np.float64)), _dp(out))
            scale_l = max(np.abs(ref[k, :3]).max(), 1e-30)
            el = np.abs(out[:3] - ref[k, :3]).max() / scale_l
            ev = np.abs(out[3:] - ref[k, 3:]).max()  # unit vectors, same sign convention
            worst = max(worst, el, ev if scale_l > 1e-6 else 0.0)
        assert worst < tol, (prec, worst)


def test_eigen_solver_right_handed_orthonormal(oracle_lib, gold):
    L = oracle_lib.lib()
    out = np.zeros(12)
    for a in gold["eig_in"][400:800]:
        L.orc_solve_eigen(64, _dp(a.astype(np.float64)), _dp(out))
        E = out[3:].reshape(3, 3)
        np.testing.assert_allclose(E @ E.T, np.eye(3), atol=1e-10)
        assert np.linalg.det(E) > 0
        assert out[0] <= out[1] + 1e-12 and out[1] <= out[2] + 1e-12


def test_johnson_cook_yield(oracle_lib, gold):
    L = oracle_lib.lib()
    jc = gold["jc"].astype(np.float64)
    got = np.array([L.orc_sigma_yield(32, _dp(jc), *row) for row in gold["jc_in"]])
    np.testing.assert_allclose(got, gold["jc_sy"], rtol=1e-12, atol=0)


def test_johnson_cook_secant(oracle_lib, gold):
    L = oracle_lib.lib()
    jc = gold["jc"].astype(np.float64)
    G, dt = float(gold["secant_G"]), float(gold["secant_dt"])
    f = C.c_int()
    for k, (normS, eps0, T, epsd) in enumerate(gold["secant_in"]):
        init = max(epsd * dt * np.sqrt(2.0 / 3.0), 1e-8)
        r = L.orc_solve_secant(32, _dp(jc), init, 1e-6, normS, eps0, T, dt, G, 100, C.byref(f))
        assert f.value == gold["secant_fail"][k]
        assert r == pytest.approx(gold["secant_out"][k], rel=1e-12, abs=1e-15)
