"""Pin the CPU oracle to the reference's own NumPy core (golden vectors made by
tests/golden/make_golden.py from reproduction/core.py)."""
import hashlib

import numpy as np
import pytest

from oracle import hsc_oracle as O
from hsc_reimpl_b200.systems import from_dense_fixture

STIFF = ("1e+02", "1e+04", "1e+06")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("tag", STIFF)
def test_aca_matches_core(golden, tag):
    g = golden["manufactured"]
    E = g[f"{tag}/E"]
    U, V, res, piv = O.aca(E, max_rank=min(E.shape))
    assert np.array_equal(np.asarray([p[:2] for p in piv]), g[f"{tag}/aca/pivots"])
    assert U.shape == g[f"{tag}/aca/U"].shape
    assert np.max(np.abs(U - g[f"{tag}/aca/U"])) <= 1e-12 * np.max(np.abs(U))
    assert np.max(np.abs(V - g[f"{tag}/aca/V"])) <= 1e-12 * np.max(np.abs(V))
    assert np.allclose(res, g[f"{tag}/aca/residuals"], rtol=1e-9, atol=1e-15)


@pytest.mark.parametrize("tag", STIFF)
@pytest.mark.parametrize("order", (1, 3, 5, 8))
def test_affine_neumann_matches_core(golden, tag, order):
    g = golden["manufactured"]
    P = O.neumann_dense(g[f"{tag}/A"], 12, order, 0.7)
    Pg = g[f"{tag}/o{order}/P"]
    assert np.max(np.abs(P - Pg)) <= 1e-12 * np.max(np.abs(Pg))


@pytest.mark.parametrize("tag", STIFF)
@pytest.mark.parametrize("order", (1, 3, 5, 8))
def test_hsc_solve_matches_core(golden, tag, order):
    """Same algorithm on the 216-dof fixtures: iterations within one of
    core.py (which tests the true residual every iteration) and the solution
    to the PCG tolerance."""
    g = golden["manufactured"]
    D, A, E, b = (g[f"{tag}/{k}"] for k in "DAEb")
    s = from_dense_fixture(D, A, E, b)
    x, st, orc = O.hsc_solve(s.H, s.layout, s.b, order=order, omega=0.7, tol=1e-10,
                             max_iter=1000, abd_inverse="neumann", max_rank=36)
    assert abs(st["pcg_iterations"] - int(g[f"{tag}/o{order}/iterations"])) <= 1
    assert rel(orc.C, g[f"{tag}/o{order}/C"]) < 1e-11
    assert rel(x, g[f"{tag}/o{order}/x"]) < 1e-7


@pytest.mark.parametrize("tag", STIFF)
def test_exact_affine_matches_core_and_direct(golden, tag):
    g = golden["manufactured"]
    D, A, E, b = (g[f"{tag}/{k}"] for k in "DAEb")
    s = from_dense_fixture(D, A, E, b)
    x, st, _ = O.hsc_solve(s.H, s.layout, s.b, order=5, omega=0.7, tol=1e-10,
                           max_iter=1000, abd_inverse="exact", max_rank=36)
    assert abs(st["pcg_iterations"] - int(g[f"{tag}/exact/iterations"])) <= 1
    assert rel(x, g[f"{tag}/exact/x"]) < 1e-7
    assert rel(x, g[f"{tag}/x_direct"]) < 1e-6


def test_numerical_checks_of_reference(golden):
    """The 13 checks of reproduction/run.py:70-107 against this restatement."""
    c = golden["checks"]
    E = c["aca_E"]
    U, V, res, _ = O.aca(E, rtol=1e-12)
    assert U.shape[1] == int(c["aca_rank"]) == 4
    assert rel(U @ V.T, E) <= 1e-12
    assert np.max(np.abs(U - c["aca_U"])) < 1e-12 * np.max(np.abs(U))
    assert O.aca(E, max_rank=3)[0].shape[1] == int(c["aca_fixed3_rank"]) == 3
    assert O.aca(np.zeros((12, 30)))[0].shape[1] == 0
    A = c["neumann_A"]
    M = O.neumann_dense(A, 12, 5, 0.7)
    Mg = c["neumann_M"]
    assert np.max(np.abs(M - Mg)) < 1e-12
    T = np.eye(24) - 0.7 * np.kron(np.eye(2), np.eye(12)) @ np.block(
        [[np.linalg.inv(A[:12, :12]), np.zeros((12, 12))], [np.zeros((12, 12)), np.linalg.inv(A[12:, 12:])]]) @ A
    assert np.max(np.abs(np.eye(24) - M @ A - np.linalg.matrix_power(T, 5))) < 1e-12
    assert np.max(np.abs(M - M.T)) < 1e-12
    s = from_dense_fixture(c["small_D"], c["small_A"], c["small_E"], c["small_b"])
    x, st, orc = O.hsc_solve(s.H, s.layout, s.b, order=5, omega=0.7, tol=1e-12, max_iter=1000,
                             abd_inverse="exact", max_rank=10 ** 6)
    assert rel(x, c["small_x"]) < 1e-8
    assert rel(s.H @ x, s.b) < 1e-10
    d = c["small_direction"]
    assert rel(orc.schur(d), c["small_schur_mv"]) < 1e-12
    # zero right-hand side: zero solution, zero iterations
    x0, st0, _ = O.hsc_solve(s.H, s.layout, np.zeros_like(s.b), abd_inverse="exact")
    assert np.all(x0 == 0) and st0["pcg_iterations"] == 0


def test_cube_matches_core(golden, cube_system):
    g = golden["cube"]
    h = hashlib.sha256()
    Hc = cube_system.H.tocsr()
    Hc.sort_indices()
    for a in (Hc.indptr, Hc.indices, Hc.data, cube_system.b):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest().encode() == bytes(g["digest"]), "cube generator drifted from the golden inputs"
    s = cube_system
    qo, qm, fo, fn = s.layout

    def core_order(x):
        return np.concatenate([x[fo:fo + fn], x[qo:qo + qm]])

    x, st, orc = O.hsc_solve(s.H, s.layout, s.b, order=2, omega=2 / 3, aca_rtol=1e-4, tol=1e-6,
                             max_iter=20000, abd_inverse="neumann", max_rank=10 ** 6)
    assert orc.rank == int(g["o2/rank"])
    assert np.allclose(orc.aca_hist, g["o2/aca_residuals"], rtol=1e-8, atol=1e-14)
    assert abs(st["pcg_iterations"] - int(g["o2/iterations"])) <= 1
    assert rel(core_order(x), g["o2/x"]) < 1e-5
    x, st, orc = O.hsc_solve(s.H, s.layout, s.b, order=2, omega=2 / 3, aca_rtol=1e-4, tol=1e-6,
                             max_iter=20000, abd_inverse="exact", max_rank=10 ** 6)
    assert abs(st["pcg_iterations"] - int(g["exact/iterations"])) <= 1
    assert rel(core_order(x), g["exact/x"]) < 1e-5
    assert st["full_relative_residual"] < 1e-6


@pytest.mark.parametrize("drop", [False, True])
def test_uncoupled_cube_oracle(cube_system, drop):
    """No active FEM dof (every coupling block zero, or none stored): ACA returns
    rank 0 (core.py:22-50 with a zero E), dq = P b_q and the PCG runs over D alone."""
    s = cube_system
    qo, qm, fo, fn = s.layout
    qb = (s.rows < (qo + qm) // 3) != (s.cols < (qo + qm) // 3)
    rows, cols, vals = s.rows, s.cols, s.vals.copy()
    if drop:
        rows, cols, vals = rows[~qb], cols[~qb], vals[~qb]
    else:
        vals[qb] = 0.0
    H = O.full_from_bcoo(rows, cols, vals, s.nblock)
    x, st, orc = O.hsc_solve(H, s.layout, s.b, order=2, omega=2 / 3, tol=1e-6, max_iter=20000,
                             abd_inverse="exact")
    assert orc.rank == 0 and orc.active.size == 0 and orc.aca_error == 0.0
    A = H[qo:qo + qm, qo:qo + qm].toarray()
    assert rel(x[qo:qo + qm], np.linalg.solve(A, s.b[qo:qo + qm])) < 1e-8
    assert st["converged"] and st["full_relative_residual"] < 1e-5
