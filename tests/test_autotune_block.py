"""The block preconditioner's polynomial tuner (``autotune.tune_block``) and its Chebyshev weights."""
import numpy as np
import pytest

from hsc_reimpl_b200 import autotune as AT


@pytest.mark.parametrize("n,a,b,omega", [(3, 0.2, 3.9, 0.5), (5, 0.4, 3.9, 0.5), (6, 0.5, 4.2, 0.6)])
def test_chebyshev_weights_give_the_chebyshev_residual_polynomial(n, a, b, omega):
    """omega lambda sum_k w_k (1 - omega lambda)^k = 1 - T_n((b + a - 2 lambda)/(b - a)) / T_n((b + a)/(b - a))."""
    from numpy.polynomial import chebyshev as Ch
    w = AT.chebyshev_weights(n, a, b, omega)
    assert len(w) == n
    lam = np.linspace(0.0, b, 97)
    p = omega * sum(wk * (1.0 - omega * lam) ** k for k, wk in enumerate(w))
    r = Ch.chebval((b + a - 2 * lam) / (b - a), [0] * n + [1]) / Ch.chebval((b + a) / (b - a), [0] * n + [1])
    np.testing.assert_allclose(lam * p, 1.0 - r, atol=1e-10)
    # on [a, b] the residual is bounded by 1 / T_n(x0): the polynomial preconditioner is SPD there
    inside = (lam >= a) & (lam <= b)
    assert np.all(np.abs(r[inside]) <= 1.0 / Ch.chebval((b + a) / (b - a), [0] * n + [1]) + 1e-12)


def test_block_candidates_include_the_reference_series():
    names = [c[0] for c in AT.block_candidates()]
    assert "neumann4 omega=0.5" in names
    for name, w, om in AT.block_candidates():
        assert 0 < om <= 1 and 1 <= len(w) <= 16


@pytest.mark.gpu
def test_tune_block_picks_a_converged_candidate_no_slower_than_neumann4():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200.systems import make_reference_vehicle_system
    s = make_reference_vehicle_system(0)
    cands = [("neumann4 omega=0.5", [1.0] * 4, 0.5), ("cheb6 a=0.5", AT.chebyshev_weights(6, 0.5, 3.9, 0.5), 0.5),
             ("neumann3 omega=0.7", [1.0] * 3, 0.7)]
    best, table = AT.tune_block(s, candidates=cands, reps=2)
    assert best is not None and len(table) == 3
    ok = [r for r in table if r["ok"]]
    assert ok, table
    # the fastest, or among those within 1 % of it the one with the fewest iterations
    fastest = min(r["ms"] for r in ok)
    chosen = min((r for r in ok if r["ms"] <= 1.01 * fastest), key=lambda r: (r["iterations"], r["ms"]))
    assert np.allclose(best.poly_weights, chosen["weights"], rtol=1e-5) and best.omega == chosen["omega"]
    assert chosen["ms"] <= 1.01 * next(r["ms"] for r in table if r["name"] == "neumann4 omega=0.5")
