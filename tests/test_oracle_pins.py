"""Pins of the two oracles that are not restatements of core.py.

* FEM Hessian (``oracle/fem_oracle.py``): the reference pins its log-Neo-Hookean
  derivatives by central differences (``reproduction/hsc_backend/check_log_nh.cpp:52-78``):
  32 deformation gradients F = I + N(0, 0.12) per entry from an MT19937 seeded 718
  (the first one scaled by 0.35, a strong feasible compression), mu = 3.2,
  lambda = 4.7, h = 1e-6; the gradient against differences of the energy and every
  Hessian column against differences of the gradient must agree to 1e-7 (relative to
  1 + norm), the projected Hessian must be positive semi-definite (smallest
  eigenvalue >= -1e-8) and equal to the eigenvalue-clamped raw Hessian.  The same
  method and bounds are used here; numpy's MT19937 draws the normals through its own
  transform, so the 32 samples are not the reference's bit for bit.
* Coupling Jacobian (``oracle/coupling_oracle.py``): ``jacobian(xbar, p_first=False)``
  against ``core.affine_projection`` (``reproduction/core.py:201-206``) at 64 seeded
  rest points, saved by ``tests/golden/make_golden.py``.
"""
import numpy as np

from oracle import coupling_oracle as CO
from oracle import fem_oracle as FO
from tests.conftest import GOLDEN


def _samples():
    rng = np.random.RandomState(718)
    Fs = []
    for s in range(32):
        F = np.eye(3) + rng.normal(0.0, 0.12, size=(3, 3))
        if s == 0:
            F *= 0.35
        Fs.append(F)
    return np.stack(Fs)


def _vec(F):
    """column-major vec of a 3x3 matrix (Eigen's data() order)."""
    return F.T.reshape(9)


def test_log_nh_derivatives_match_central_differences():
    mu, lam, h = 3.2, 4.7, 1e-6
    Fs = _samples()
    m, l = np.full(1, mu), np.full(1, lam)
    max_g = max_h = 0.0
    for F in Fs:
        P = FO.first_piola(F[None], m, l)[0]
        H = FO.raw_hessian(F[None], m, l)[0]
        for k in range(9):
            d = np.zeros(9)
            d[k] = h
            dF = d.reshape(3, 3).T                        # column-major entry k
            ep = FO.energy((F + dF)[None], m, l)[0]
            em = FO.energy((F - dF)[None], m, l)[0]
            max_g = max(max_g, abs((ep - em) / (2 * h) - _vec(P)[k]) / (1 + np.linalg.norm(P)))
            pp = FO.first_piola((F + dF)[None], m, l)[0]
            pm = FO.first_piola((F - dF)[None], m, l)[0]
            col = _vec((pp - pm) / (2 * h))
            max_h = max(max_h, np.linalg.norm(col - H[:, k]) / (1 + np.linalg.norm(H)))
        Hs = FO.spd(H[None])[0]
        assert np.linalg.eigvalsh(Hs).min() >= -1e-8
        w, Q = np.linalg.eigh(H)
        expected = Q @ np.diag(np.maximum(w, 0.0)) @ Q.T
        assert np.linalg.norm(Hs - expected) / (1 + np.linalg.norm(expected)) <= 1e-9
    assert max_g <= 1e-7, max_g
    assert max_h <= 1e-7, max_h


def test_log_nh_energy_is_infinite_for_inverted_F():
    F = np.eye(3)
    F[2, 2] = -1.0
    assert np.isinf(FO.energy(F[None], np.full(1, 3.2), np.full(1, 4.7))[0])


def test_coupling_jacobian_matches_core_affine_projection():
    g = np.load(GOLDEN / "projection.npz")
    for rest, P in zip(g["rest"], g["P"]):
        np.testing.assert_array_equal(CO.jacobian(rest, p_first=False), P)
    # libuipc's (p, rows of A) order is the same map with the columns permuted
    perm = np.r_[9:12, 0:9]
    for rest, P in zip(g["rest"], g["P"]):
        np.testing.assert_array_equal(CO.jacobian(rest, p_first=True), P[:, perm])


def test_systems_affine_projection_matches_core():
    from hsc_reimpl_b200.systems import affine_projection
    g = np.load(GOLDEN / "projection.npz")
    for rest, P in zip(g["rest"], g["P"]):
        np.testing.assert_array_equal(affine_projection(rest), P)
