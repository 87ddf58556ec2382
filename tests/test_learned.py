"""Learned polynomial preconditioner: the CPU oracle (finite-difference
gradient checks, the least-squares teacher), the training-system generator,
and -- on the GPU, through the C ABI -- the MLP / loss / Adam kernels, the
device features and the Schur-basis polynomial solve against the oracle,
the fallback, training, and what the trained model gains over the plain
Neumann series."""
import numpy as np
import pytest

from oracle import hsc_oracle as O
from oracle import learned_oracle as LO

RNG = np.random.default_rng(5)


def random_params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, scale, LO.NPARAM).astype(np.float32)
    bits = LO.bf16_round(p)
    return bits, LO.bf16_to_float(bits)


def random_batch(B=64, m=16, seed=1):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (B, LO.NF)).astype(np.float32)
    th = np.sort(rng.uniform(1e-4, 1.7, (B, m)), axis=1).astype(np.float32)
    tau = rng.uniform(0, 1, (B, m))
    tau = (tau / tau.sum(1, keepdims=True)).astype(np.float32)
    return X, th, tau


# ---------------------------------------------------------------------------
# CPU: the oracle itself
# ---------------------------------------------------------------------------
def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], np.float32)
    got = LO.bf16_to_float(LO.bf16_round(x))
    assert got[0] == 1.0 and got[1] == 1.0          # tie -> even mantissa
    assert got[2] == np.float32(1.0 + 2 ** -7)      # above the tie -> up
    assert got[3] == -2.5
    assert abs(got[4] - 3e-3) / 3e-3 < 2 ** -8


def test_oracle_gradients_match_finite_differences():
    _, p = random_params(3)
    X, th, tau = random_batch(B=8, seed=4)
    X, th, tau = X.astype(np.float64), th.astype(np.float64), tau.astype(np.float64)

    def total(pp):
        w = LO.mlp_forward(pp, X)[3]
        return LO.poly_ls_loss(w, th, tau)[0].sum()

    h1, h2, o, w = LO.mlp_forward(p, X)
    _, gw = LO.poly_ls_loss(w, th, tau)
    g = LO.mlp_backward(p, X, h1, h2, o, gw)
    idx = RNG.choice(LO.NPARAM, 40, replace=False)
    for i in idx:
        e = np.zeros(LO.NPARAM)
        e[i] = 1e-6
        fd = (total(p + e) - total(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])) + 1e-7, (i, fd, g[i])


def test_loss_gradient_in_w_matches_finite_differences():
    X, th, tau = random_batch(B=4, seed=6)
    w = RNG.uniform(0.1, 3.0, (4, LO.NO))
    _, gw = LO.poly_ls_loss(w, th.astype(np.float64), tau.astype(np.float64))
    for k in range(LO.NO):
        e = np.zeros_like(w)
        e[:, k] = 1e-7
        fd = (LO.poly_ls_loss(w + e, th, tau)[0] - LO.poly_ls_loss(w - e, th, tau)[0]) / 2e-7
        assert np.allclose(fd, gw[:, k], rtol=1e-5, atol=1e-8)


def test_ls_teacher_beats_neumann_on_its_measure():
    th = np.concatenate([np.geomspace(1e-4, 0.1, 10), np.linspace(0.2, 1.6, 6)])
    tau = np.full(th.size, 1.0 / th.size)
    w = LO.ls_teacher(th, tau)
    assert np.all(w >= 0)
    lt = LO.poly_ls_loss(w[None], th[None], tau[None])[0][0]
    ln = LO.poly_ls_loss(np.ones((1, LO.NO)), th[None], tau[None])[0][0]
    assert lt < ln


def test_lanczos_measure_reproduces_spectrum():
    # CG on a diagonal matrix: the full Lanczos measure is the spectrum with
    # weights = squared components of the normalised start vector
    lam = np.array([0.01, 0.1, 0.5, 1.0, 1.5])
    b = np.array([1.0, 2.0, 0.5, 1.0, 3.0])
    A = np.diag(lam)
    _, st = O.pcg_schur(lambda p: A @ p, b, lambda r: r.copy(), 1e-14, 5)
    th, tau = LO.lanczos_measure(st["alphas"], st["betas"] + [0.0], 5)
    assert np.allclose(np.sort(th), lam, rtol=1e-8)
    assert np.allclose(tau[np.argsort(th)], b ** 2 / (b @ b), rtol=1e-6)


def test_schur_basis_oracle_is_polynomial_in_schur_operator():
    from hsc_reimpl_b200.systems import make_cube_system
    s = make_cube_system(seed=0)
    orc = O.HSCOracle(s.H, s.layout, order=3, omega=2 / 3, basis="schur", weights=[1.0, 0.5, 2.0],
                      abd_inverse="exact", aca_rtol=1e-4)
    r = RNG.standard_normal(s.layout[3])
    z = orc.precond(r)
    # explicit: G = w Dd^-1 S applied as a matrix polynomial to t0 = w Dd^-1 r
    t0 = (2 / 3) * O.block_diag_apply(orc.Dinv, r)
    G = lambda v: (2 / 3) * O.block_diag_apply(orc.Dinv, orc.schur(v))
    t1 = t0 - G(t0)
    t2 = t1 - G(t1)
    assert np.allclose(z, t0 + 0.5 * t1 + 2.0 * t2, rtol=1e-12, atol=1e-14)


@pytest.mark.slow
def test_trajectory_matches_independent_assembly():
    """The fast trajectory generator (fixed parts reduced once, contacts per
    step) equals a from-scratch assembly of the same vehicle system."""
    from hsc_reimpl_b200 import learned as L
    from hsc_reimpl_b200 import systems as S
    B = L.VehicleBase(0)
    steps = list(L.VehicleTrajectory(B, seed=3, steps=12, contact_every=10))
    _, rows, cols, vals, meta = steps[11]
    assert np.all(np.diff(rows.astype(np.int64) * B.nblock + cols) > 0)   # sorted, unique, one triangle
    assert np.all(rows <= cols)
    H = O.full_from_bcoo(rows, cols, np.transpose(vals.reshape(-1, 3, 3), (0, 2, 1)), B.nblock)
    rng = np.random.default_rng(10_000)
    qm, fn = B.qm, B.fn
    asm = S._Assembler(qm + fn)
    nr, na, nc = 4, 5, 93
    for t in range(7):
        center = np.array([1.2 * (t % 4), 0.5 * (t // 4), 0.0])
        x, tets, _ = S.annulus_mesh(nr=nr, na=na, nc=nc, center=center)
        base = t * B.nodes_per
        r, c, v, _ = S.fem_hessian(x, tets, meta["E"][t], 0.3, 1000.0, perturb=0.02, rng=rng)
        asm.add(qm + 3 * base + r, qm + 3 * base + c, v)
        rim = [((0 * (na + 1) + ia) * nc + ic) for ia in (0, na) for ic in range(0, nc, 5)]
        asm.add_dense(12 * t + np.arange(12), S.abd_block(20.0, x[rim] - center, 1e10, np.pi * 0.27 ** 2 * 0.3 * 0.1))
        for node in rim:
            S._stitch(asm, qm, base + node, t, x[node] - center, 1e7)
    for s in range(4):
        pts = rng.uniform(-0.1, 0.1, (16, 3))
        asm.add_dense(12 * (7 + s) + np.arange(12), S.abd_block(10.0, pts, 1e10, 0.004))
        for p in (np.array([0.0, 0.1, 0.0]), np.array([0.05, 0.1, 0.05]), np.array([0.0, 0.1, 0.08])):
            S._joint(asm, 7 + s, p, s, p + np.array([0.0, -0.25, 0.0]), 1e9)
    for s in range(3):
        S._joint(asm, 7 + s, np.array([0.3, 0.0, 0.0]), 8 + s, np.array([-0.3, 0.0, 0.0]), 1e7)
    gpts = rng.uniform(-2.0, 2.0, (32, 3))
    asm.add_dense(12 * 11 + np.arange(12), S.abd_block(1e4, gpts, 1e10, 10.0))
    for node, nv, k in zip(meta["contact_nodes"], meta["normals"], meta["k"]):
        S._barrier_coupling(asm, qm, node, 11, B.x[node] - B.ground_point, nv, k)
    Href = asm.csr()
    d = H - Href
    assert np.sqrt(d.multiply(d).sum()) <= 1e-13 * np.sqrt(Href.multiply(Href).sum())
    assert 6.0 <= np.log10(meta["E"][4:]).min() and np.log10(meta["E"][4:]).max() <= 8.0


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def api(torch):
    from hsc_reimpl_b200 import solver
    return solver


def _dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


@pytest.mark.gpu
def test_mlp_training_kernels_match_oracle(torch):
    from hsc_reimpl_b200 import learned as L
    bits, p = random_params(11)
    X, th, tau = random_batch(B=300, seed=12)
    tr = L.Trainer(L.bf16_values(bits))
    assert np.array_equal(tr.pbf.cpu().numpy().view(np.uint16), bits)
    Xd, THd, TAUd = _dev(torch, X), _dev(torch, th), _dev(torch, tau)
    w = tr.forward(Xd, 300).cpu().numpy()
    h1, h2, o, w_ref = LO.mlp_forward(p, X)
    assert np.allclose(w, w_ref, rtol=2e-5, atol=1e-6)
    assert np.allclose(tr.h1[:300].cpu().numpy(), h1, rtol=2e-5, atol=1e-5)
    loss = tr.loss_and_grad(Xd, THd, TAUd).cpu().numpy()
    loss_ref, gw_ref = LO.poly_ls_loss(w_ref, th.astype(np.float64), tau.astype(np.float64), scale=1 / 300)
    assert np.allclose(loss, loss_ref, rtol=1e-4, atol=1e-7)
    assert np.allclose(tr.gw[:300].cpu().numpy(), gw_ref, rtol=1e-4, atol=1e-7)
    g = tr.grad.cpu().numpy()
    g_ref = LO.mlp_backward(p, X, h1, h2, o, gw_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    # Adam: first step moves every parameter with a nonzero gradient by lr * sign(g)
    master0 = tr.master.cpu().numpy().copy()
    tr.lr = 1e-3
    tr.step(Xd, THd, TAUd)
    moved = tr.master.cpu().numpy() - master0
    nz = np.abs(g) > 1e-6
    assert np.allclose(moved[nz], -1e-3 * np.sign(g[nz]), rtol=1e-3)
    assert np.array_equal(tr.pbf.cpu().numpy().view(np.uint16), LO.bf16_round(tr.master.cpu().numpy()))


@pytest.mark.gpu
def test_training_is_deterministic_and_reduces_loss(torch):
    from hsc_reimpl_b200 import learned as L
    rng = np.random.default_rng(21)
    n = 2048
    X = rng.normal(0, 1, (n, LO.NF)).astype(np.float32)
    # the spectrum's lower edge depends on a feature: something to learn
    lo = 10.0 ** (-3 + X[:, 0:1].clip(-1, 1))
    th = np.concatenate([lo * np.geomspace(1, 30, 8)[None], np.linspace(0.3, 1.6, 8)[None].repeat(n, 0)], 1)
    tau = np.full(th.shape, 1.0 / th.shape[1])
    data = dict(features=X, theta=th.astype(np.float32), tau=tau.astype(np.float32))
    runs = []
    for _ in range(2):
        tr = L.Trainer(L.init_params(0), lr=3e-3, seed=0)
        l0 = tr.evaluate_loss(data)
        tr.fit(data, epochs=15, batch=256)
        runs.append((l0, tr.evaluate_loss(data), tr.params_fp32()))
    # the per-sample optimum (non-negative least squares) bounds the loss from below:
    # training closes more than half of the gap from the Neumann start to it
    best = np.mean([LO.poly_ls_loss(LO.ls_teacher(th[i], tau[i])[None], th[i:i + 1], tau[i:i + 1])[0][0]
                    for i in range(0, n, 16)])
    l0, l1 = runs[1][0], runs[1][1]
    assert l1 - best < 0.5 * (l0 - best), (l0, l1, best)
    assert np.array_equal(runs[0][2], runs[1][2])


def _cube(api):
    from hsc_reimpl_b200.systems import make_cube_system
    s = make_cube_system(seed=0)
    return s, api.DeviceSystem.from_system(s)


@pytest.mark.gpu
# weights whose polynomial q stays positive on (0, 2] (an SPD preconditioner for the cube)
@pytest.mark.parametrize("weights", [(1.0, 1.0, 1.0, 1.0), (1.0, 1.0, 0.5, 0.25), tuple(0.9 ** k for k in range(8))])
def test_schur_polynomial_solve_matches_oracle(api, torch, weights):
    s, ds = _cube(api)
    o = dict(omega=2 / 3, aca_rtol=1e-4, tol=1e-6)
    ctx = api.HSCContext(api.HSCOptions(poly_weights=weights, poly_basis="schur", abd_inverse="exact", **o))
    x, st = ctx.solve(ds)
    xr, sr, _ = O.hsc_solve(s.H, s.layout, s.b, order=len(weights), weights=list(weights), basis="schur",
                            abd_inverse="exact", max_iter=20000, **o)
    assert st["fallback"] == 0
    assert abs(st["pcg_iterations"] - sr["pcg_iterations"]) <= 1
    xs = x.cpu().numpy()
    assert np.linalg.norm(xs - xr) <= 1e-5 * np.linalg.norm(xr)
    assert st["full_relative_residual"] <= 1e-5


@pytest.mark.gpu
def test_schur_polynomial_vehicle_fewer_iterations(api, torch, vehicle_system):
    s = vehicle_system
    ds = api.DeviceSystem.from_system(s)
    ctx = api.HSCContext(api.HSCOptions(neumann_order=2))
    _, st2 = ctx.solve(ds)
    ctx.set_options(api.HSCOptions(poly_weights=(1.0,) * 8, poly_basis="schur"))
    x, st8 = ctx.solve(ds)
    xs = x.cpu().numpy()
    assert np.linalg.norm(s.H @ xs - s.b) <= 1e-6 * np.linalg.norm(s.b) * 1.01
    assert st8["pcg_iterations"] < 0.7 * st2["pcg_iterations"]
    # the same weights on the FEM-basis terms barely help (the coupled modes live in S)
    ctx.set_options(api.HSCOptions(poly_weights=(1.0,) * 8, poly_basis="fem"))
    _, stf = ctx.solve(ds)
    assert st8["pcg_iterations"] < stf["pcg_iterations"]


@pytest.mark.gpu
def test_device_features_match_oracle(api, torch):
    s, ds = _cube(api)
    opts = dict(omega=2 / 3, aca_rtol=1e-4, abd_inverse="exact")
    ctx = api.HSCContext(api.HSCOptions(lanczos_stats=True, **opts))
    _, st = ctx.solve(ds)
    f1 = ctx.features()
    orc = O.HSCOracle(s.H, s.layout, order=2, **opts)
    ref = LO.features(orc.D, s.layout, orc.active, orc.V, orc.C, prev=None)
    assert np.allclose(f1, ref, rtol=1e-5, atol=1e-6), (f1, ref)
    assert f1[12] == 0.0
    # the second solve sees the first one's Lanczos record
    _, st2 = ctx.solve(ds)
    f2 = ctx.features()
    ref2 = LO.features(orc.D, s.layout, orc.active, orc.V, orc.C,
                       prev=(st["lanczos_min"], st["lanczos_max"], st["pcg_iterations"], 2.0))
    assert np.allclose(f2, ref2, rtol=1e-5, atol=1e-6), (f2, ref2)
    assert f2[12] == 1.0


@pytest.mark.gpu
def test_learned_solve_uses_model_weights(api, torch):
    s, ds = _cube(api)
    bits, p = random_params(31, scale=0.1)
    opts = dict(omega=2 / 3, aca_rtol=1e-4, abd_inverse="exact", tol=1e-6)
    ctx = api.HSCContext(api.HSCOptions(learned=True, **opts))
    ctx.set_learned_model(bits)
    x, st = ctx.solve(ds)
    f = ctx.features()
    w = ctx.poly_weights()
    w_ref = LO.mlp_forward(p, f[None].astype(np.float64))[3][0]
    assert w.size == 8 and np.allclose(w, w_ref, rtol=1e-5)
    assert st["fallback"] == 0 and st["status"] == 0
    xr, sr, _ = O.hsc_solve(s.H, s.layout, s.b, order=8, weights=list(w), basis="schur", max_iter=20000, **opts)
    assert abs(st["pcg_iterations"] - sr["pcg_iterations"]) <= 1
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-5 * np.linalg.norm(xr)


@pytest.mark.gpu
def test_learned_without_model_is_rejected(api, torch):
    _, ds = _cube(api)
    ctx = api.HSCContext(api.HSCOptions(learned=True))
    from hsc_reimpl_b200._lib import HSCError
    with pytest.raises(HSCError, match="invalid"):
        ctx.solve(ds)


@pytest.mark.gpu
def test_learned_falls_back_to_neumann_on_stall(api, torch):
    s, ds = _cube(api)
    bits, _ = random_params(41, scale=0.1)
    opts = dict(omega=2 / 3, aca_rtol=1e-4, abd_inverse="exact")
    ctx = api.HSCContext(api.HSCOptions(learned=True, max_iter=3, **opts))
    ctx.set_learned_model(bits)
    _, st = ctx.solve(ds, raise_on_error=False)
    assert st["fallback"] == 1
    assert st["status_name"] == "noconv"           # the Neumann redo also stops at max_iter
    # a model whose polynomial is negative above mu = 1 (indefinite): the redo converges
    p = np.zeros(LO.NPARAM, np.float32)
    w_bad = np.array([1e-3, 0, 0, 0, 0, 0, 0, 1e5])
    wb = np.maximum(w_bad, 1e-12)
    p[LO.OFF_B3:] = np.where(wb > 20, wb, np.log(np.expm1(np.minimum(wb, 20))))
    ctx2 = api.HSCContext(api.HSCOptions(learned=True, **opts))
    ctx2.set_learned_model(LO.bf16_round(p))
    x, st2 = ctx2.solve(ds, raise_on_error=False)
    assert st2["status"] == 0
    if st2["fallback"]:
        assert st2["preconditioner"] == 0
    assert np.linalg.norm(s.H @ x.cpu().numpy() - s.b) <= 1e-5 * np.linalg.norm(s.b)


@pytest.mark.gpu
def test_trained_model_beats_neumann_on_held_out_vehicle_steps(api, torch):
    from hsc_reimpl_b200 import learned as L
    if not L.MODEL_PATH.exists():
        pytest.skip("no trained model file")
    bits, meta = L.load_model()
    base = L.VehicleBase(meta.get("eval_variant", 3))
    traj = L.VehicleTrajectory(base, seed=meta.get("eval_seeds", [9001])[0], steps=6)
    res = L.evaluate(bits, [traj])
    n2, n8, le = (res[k]["iters"].mean() for k in ("neumann2", "schur_neumann8", "learned"))
    assert np.all(res["learned"]["full"] <= 1e-6 * 1.01)
    assert le < 0.7 * n2
    assert le < n8


@pytest.mark.gpu
def test_learned_batch_falls_back_per_system(api, torch):
    """In a batch, the systems whose learned polynomial stalls are solved again with the plain
    Neumann series (a sub-batch); their stats say so and carry the iterations of both attempts."""
    s, ds = _cube(api)
    opts = dict(omega=2 / 3, aca_rtol=1e-4, abd_inverse="exact")
    bits, _ = random_params(41, scale=0.1)
    ctx = api.HSCContext(api.HSCOptions(learned=True, max_iter=3, **opts))
    ctx.set_learned_model(bits)
    _, sts = ctx.solve_batch([ds, ds], raise_on_error=False)
    from hsc_reimpl_b200 import _lib
    for st in sts:
        assert st["fallback"] == 1 and st["status"] == _lib.HSC_ERR_NOCONV  # the redo also stops at max_iter
    # an indefinite polynomial (negative above mu = 1): every system ends converged
    p = np.zeros(LO.NPARAM, np.float32)
    w_bad = np.array([1e-3, 0, 0, 0, 0, 0, 0, 1e5])
    wb = np.maximum(w_bad, 1e-12)
    p[LO.OFF_B3:] = np.where(wb > 20, wb, np.log(np.expm1(np.minimum(wb, 20))))
    ctx2 = api.HSCContext(api.HSCOptions(learned=True, **opts))
    ctx2.set_learned_model(LO.bf16_round(p))
    xs, sts = ctx2.solve_batch([ds, ds], raise_on_error=False)
    for x, st in zip(xs, sts):
        assert st["status"] == 0
        assert np.linalg.norm(s.H @ x.cpu().numpy() - s.b) <= 1e-5 * np.linalg.norm(s.b)
