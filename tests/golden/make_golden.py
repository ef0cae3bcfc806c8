"""Generate tests/golden/ref_kat.npz from the reference's own functions.

Inputs are seeded; outputs come from oracle/_ref/libref_kat.so, i.e. the
reference's cubic_spline / lapl_pse (src/kernels.cuh), solve_eigen
(src/eigen_solver.cu) and sigma_yield / solve_secant (src/plasticity.cuh)
compiled unchanged for the host by oracle/build_ref.sh.  Run in a checkout that
has the reference sources:  python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402


def main():
    oracle.build_ref()
    R = oracle.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libref_kat.so is missing (reference sources not found)")
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    rng = np.random.default_rng(20240601)
    h = np.float32(1.3e-3)
    # kernel function: pairs inside, near and outside the support, and coincident
    n = 4000
    pi = rng.uniform(-2e-3, 2e-3, (n, 3)).astype(np.float32)
    d = rng.uniform(-3.2e-3, 3.2e-3, (n, 3))
    d[:50] = 0.0
    d[50:100] *= 1e-4
    pj = (pi + d).astype(np.float32)
    hs = np.full(n, h, np.float32)
    hs[::7] = np.float32(1.7e-3)
    w = np.zeros((n, 4), np.float32)
    pse = np.zeros(n, np.float32)
    for k in range(n):
        out = np.zeros(4, np.float32)
        R.ref_cubic_spline(fp(pi[k].copy()), fp(pj[k].copy()), hs[k], fp(out))
        w[k] = out
        pse[k] = R.ref_lapl_pse(fp(pi[k].copy()), fp(pj[k].copy()), hs[k])
    # eigen solver: random symmetric, diagonal, tiny, repeated-eigenvalue and stress-like matrices
    m = 3000
    A = rng.normal(size=(m, 6)).astype(np.float32) * np.float32(1e-2)
    A[:100, 1] = A[:100, 2] = A[:100, 4] = 0          # diagonal
    A[100:150] *= np.float32(1e-7)                      # below 1e-8 after scaling? (tiny)
    A[150:250] = np.array([1, 0, 0, 1, 0, 1], np.float32) * rng.normal(size=(100, 1)).astype(np.float32)
    A[250:400, 0] = A[250:400, 3]                       # partly repeated
    eig = np.zeros((m, 12), np.float32)
    for k in range(m):
        out = np.zeros(12, np.float32)
        R.ref_solve_eigen(fp(A[k].copy()), fp(out))
        eig[k] = out
    # Johnson-Cook
    jc = np.array([7.92e-3, 5.10e-3, 0.014, 0.26, 1.03, 1793.0, 300.0, 1e-6, 1.0], np.float32)
    q = 2000
    jin = np.stack([rng.uniform(0, 0.6, q), 10 ** rng.uniform(-10, -2, q), rng.uniform(300, 1700, q)], 1)
    jin[:20, 1] = 0.0
    sy = np.array([R.ref_sigma_yield(fp(jc), *row) for row in jin])
    # secant: trial stress norms above yield, the reference's tolerance and start value
    s = 500
    G = 0.7751938
    dt = 4.0467537e-4
    sin = np.stack([rng.uniform(0.005, 0.02, s), rng.uniform(0, 0.3, s), rng.uniform(300, 1200, s),
                    10 ** rng.uniform(-8, -3, s)], 1)
    sec = np.zeros(s)
    fail = np.zeros(s, np.int32)
    for k in range(s):
        normS, eps0, T, epsd = sin[k]
        init = max(epsd * dt * np.sqrt(2.0 / 3.0), 1e-8)
        f = C.c_int()
        sec[k] = R.ref_solve_secant(fp(jc), init, 1e-6, normS, eps0, T, dt, G, C.byref(f))
        fail[k] = f.value
    np.savez_compressed(os.path.join(HERE, "ref_kat.npz"), spline_pi=pi, spline_pj=pj, spline_h=hs, spline_w=w,
                        pse=pse, eig_in=A, eig_out=eig, jc=jc, jc_in=jin, jc_sy=sy, secant_in=sin, secant_G=G,
                        secant_dt=dt, secant_out=sec, secant_fail=fail)
    print("wrote", os.path.join(HERE, "ref_kat.npz"))


if __name__ == "__main__":
    main()
