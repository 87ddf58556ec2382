"""GPU parity of the CUDA HSC path against the CPU oracle and the reference's
golden vectors, through the C ABI (hsc_solve / hsc_spmv / hsc_get_*)."""
import numpy as np
import pytest

from oracle import hsc_oracle as O
from hsc_reimpl_b200 import systems as S

pytestmark = pytest.mark.gpu

STIFF = ("1e+02", "1e+04", "1e+06")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


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


def fixture_system(golden, tag):
    g = golden["manufactured"]
    return S.from_dense_fixture(g[f"{tag}/D"], g[f"{tag}/A"], g[f"{tag}/E"], g[f"{tag}/b"])


# ---------------------------------------------------------------------------
# kernels
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("tag", STIFF)
def test_full_spmv_matches_dense(api, torch, golden, tag):
    """hsc_spmv (IterativeSolver::spmv) against H @ x of the reference fixture."""
    s = fixture_system(golden, tag)
    ctx = api.HSCContext()
    ds = api.DeviceSystem.from_system(s)
    rng = np.random.default_rng(7)
    for _ in range(3):
        xv = rng.standard_normal(s.N)
        y = ctx.spmv(ds, torch.from_numpy(xv).cuda()).cpu().numpy()
        assert rel(y, s.H @ xv) < 1e-14


def test_full_spmv_vehicle(api, torch, vehicle_system):
    s = vehicle_system
    ctx = api.HSCContext()
    ds = api.DeviceSystem.from_system(s)
    xv = np.random.default_rng(3).standard_normal(s.N)
    y = ctx.spmv(ds, torch.from_numpy(xv).cuda()).cpu().numpy()
    assert rel(y, s.H @ xv) < 1e-13


@pytest.mark.parametrize("tag", STIFF)
def test_aca_factors_match_reference_core(api, torch, golden, tag):
    """Device full-pivot ACA = core.aca (same pivots, same factors)."""
    g = golden["manufactured"]
    s = fixture_system(golden, tag)
    ctx = api.HSCContext(api.HSCOptions(max_rank=36, neumann_order=5, tol=1e-10, abd_inverse="neumann"))
    ds = api.DeviceSystem.from_system(s)
    ctx.solve(ds)
    U, V, act = ctx.factors_full(36)
    Ug, Vg = g[f"{tag}/aca/U"], g[f"{tag}/aca/V"]
    assert U.shape[1] == Ug.shape[1]
    # the fixture's coupling touches a subset of FEM dofs; core's V has rows for all of them
    assert np.max(np.abs(U - Ug)) <= 1e-12 * np.max(np.abs(Ug))
    assert np.max(np.abs(V - Vg[act])) <= 1e-12 * np.max(np.abs(Vg))
    mask = np.ones(Vg.shape[0], bool)
    mask[act] = False
    assert np.all(Vg[mask] == 0)


@pytest.mark.parametrize("mode", ("components", "cluster", "grid"))
def test_aca_cluster_and_grid_kernels_match_oracle(api, torch, vehicle_system, mode):
    """The three ACA paths (per coupling component with the merged pivot order,
    16-CTA cluster in distributed shared memory, grid kernel with column strips)
    reproduce the oracle's full-pivot ACA on the vehicle coupling (144 x 1749):
    same rank, same pivots, same factors."""
    s = vehicle_system
    ctx = api.HSCContext(api.HSCOptions(aca_cluster=mode == "cluster", aca_components=mode == "components",
                                        max_rank=128))
    ds = api.DeviceSystem.from_system(s)
    ctx.solve(ds)
    U, V, act = ctx.factors_full(s.layout[1])
    D, A, E, active = O.extract(s.H, s.layout)
    Uo, Vo, hist, piv = O.aca(E, max_rank=min(128, s.layout[1], active.size))
    assert np.array_equal(act, active)
    assert U.shape == Uo.shape
    assert np.max(np.abs(U - Uo)) <= 1e-11 * np.max(np.abs(Uo))
    assert np.max(np.abs(V - Vo)) <= 1e-11 * np.max(np.abs(Vo))


def test_component_aca_is_bitwise_the_global_aca(api, torch, tire_system):
    """On the tire-mesh vehicle (8 coupling components: 7 rims and the ground) the component
    ACA's merged factors equal the global cluster ACA's bit for bit, in the same column order."""
    s = tire_system
    ds = api.DeviceSystem.from_system(s)
    out = {}
    for comp in (True, False):
        ctx = api.HSCContext(api.HSCOptions(aca_components=comp, aca_cluster=True, omega=0.5, max_rank=128))
        _, st = ctx.solve(ds)
        out[comp] = (ctx.factors_full(s.layout[1]), st["rank"])
    (U1, V1, a1), k1 = out[True]
    (U0, V0, a0), k0 = out[False]
    assert k1 == k0 == 96
    np.testing.assert_array_equal(a1, a0)
    np.testing.assert_array_equal(U1, U0)
    np.testing.assert_array_equal(V1, V0)


@pytest.mark.parametrize("tag", STIFF)
@pytest.mark.parametrize("order", (1, 3, 5, 8))
def test_abd_neumann_inverse_matches_core(api, torch, golden, tag, order):
    g = golden["manufactured"]
    s = fixture_system(golden, tag)
    ctx = api.HSCContext(api.HSCOptions(max_rank=36, neumann_order=order, tol=1e-10, abd_inverse="neumann"))
    ctx.solve(api.DeviceSystem.from_system(s), raise_on_error=False)
    P = ctx.abd_inverse(36)
    Pg = g[f"{tag}/o{order}/P"]
    assert np.max(np.abs(P - Pg)) <= 1e-11 * np.max(np.abs(Pg))


def test_abd_exact_and_adaptive_inverse(api, torch, vehicle_system):
    s = vehicle_system
    _, A, _, _ = O.extract(s.H, s.layout)
    ds = api.DeviceSystem.from_system(s)
    ctx = api.HSCContext(api.HSCOptions(abd_inverse="exact"))
    ctx.solve(ds)
    P = ctx.abd_inverse(144)
    Po, _, _ = O.abd_inverse(A, "exact")
    assert rel(P, Po) < 1e-9
    ctx2 = api.HSCContext(api.HSCOptions(abd_inverse="adaptive", neumann_order=5))
    _, st = ctx2.solve(ds, raise_on_error=False)
    Pa, d, err = O.abd_inverse(A, "adaptive", order=5, omega=0.7, tol=1e-5)
    assert st["neumann_doublings"] == d
    assert st["abd_inverse_residual"] <= 1e-5
    assert rel(ctx2.abd_inverse(144), Pa) < 1e-6


# ---------------------------------------------------------------------------
# whole solves
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("tag", STIFF)
@pytest.mark.parametrize("order", (1, 3, 5, 8))
def test_solve_matches_reference_core(api, torch, golden, tag, order):
    """HSC(D, A, E, order, omega=0.7, fixed-rank ACA).solve(b) of core.py."""
    g = golden["manufactured"]
    s = fixture_system(golden, tag)
    ctx = api.HSCContext(api.HSCOptions(max_rank=36, neumann_order=order, tol=1e-10, max_iter=1000,
                                        abd_inverse="neumann", full_residual_limit=1.0))
    x, st = ctx.solve(api.DeviceSystem.from_system(s))
    assert abs(st["pcg_iterations"] - int(g[f"{tag}/o{order}/iterations"])) <= 1
    assert rel(x.cpu().numpy(), g[f"{tag}/o{order}/x"]) < 1e-7


@pytest.mark.parametrize("tag", STIFF)
def test_exact_affine_solve_matches_direct(api, torch, golden, tag):
    g = golden["manufactured"]
    s = fixture_system(golden, tag)
    ctx = api.HSCContext(api.HSCOptions(max_rank=36, neumann_order=5, tol=1e-10, max_iter=1000))
    x, st = ctx.solve(api.DeviceSystem.from_system(s))
    assert abs(st["pcg_iterations"] - int(g[f"{tag}/exact/iterations"])) <= 1
    assert rel(x.cpu().numpy(), g[f"{tag}/x_direct"]) < 1e-6
    assert st["full_relative_residual"] < 1e-9


def test_cube_matches_reference_core(api, torch, golden, cube_system):
    g = golden["cube"]
    s = cube_system
    qo, qm, fo, fn = s.layout
    ctx = api.HSCContext(api.HSCOptions(neumann_order=2, omega=2 / 3, aca_rtol=1e-4, tol=1e-6,
                                        abd_inverse="neumann"))
    x, st = ctx.solve(api.DeviceSystem.from_system(s), raise_on_error=False)
    xs = x.cpu().numpy()
    assert st["rank"] == int(g["o2/rank"])
    assert abs(st["pcg_iterations"] - int(g["o2/iterations"])) <= 1
    assert rel(np.concatenate([xs[fo:fo + fn], xs[qo:qo + qm]]), g["o2/x"]) < 1e-5
    ctx.set_options(api.HSCOptions(neumann_order=2, omega=2 / 3, aca_rtol=1e-4, tol=1e-6, abd_inverse="exact"))
    x, st = ctx.solve(api.DeviceSystem.from_system(s))
    xs = x.cpu().numpy()
    assert abs(st["pcg_iterations"] - int(g["exact/iterations"])) <= 1
    assert rel(np.concatenate([xs[fo:fo + fn], xs[qo:qo + qm]]), g["exact/x"]) < 1e-5
    assert st["full_relative_residual"] < 1e-6


@pytest.fixture(scope="module")
def vehicle_oracle(vehicle_system):
    s = vehicle_system
    x, st, orc = O.hsc_solve(s.H, s.layout, s.b, order=2, omega=0.7, tol=1e-6, max_iter=20000,
                             abd_inverse="exact", max_rank=128)
    return x, st, orc


def test_vehicle_fp64_matches_oracle(api, torch, vehicle_system, vehicle_oracle):
    s = vehicle_system
    xo, so, orc = vehicle_oracle
    ctx = api.HSCContext(api.HSCOptions(neumann_order=2, tol=1e-6))
    x, st = ctx.solve(api.DeviceSystem.from_system(s))
    assert st["rank"] == so["rank"]
    assert st["active_fem_dofs"] == so["active_fem_dofs"]
    assert abs(st["pcg_iterations"] - so["pcg_iterations"]) <= 1
    assert rel(x.cpu().numpy(), xo) < 1e-5
    assert st["full_relative_residual"] <= 1e-6


@pytest.fixture(scope="module")
def tire_system():
    from hsc_reimpl_b200.systems import make_reference_vehicle_system
    return make_reference_vehicle_system(seed=0)


@pytest.fixture(scope="module")
def tire_oracle(tire_system):
    s = tire_system
    return O.hsc_solve(s.H, s.layout, s.b, order=2, omega=0.5, tol=1e-6, max_iter=20000,
                       abd_inverse="exact", max_rank=128)


def test_tire_mesh_vehicle_fp64_matches_oracle(api, torch, tire_system, tire_oracle):
    """The benchmark workload: the vehicle scene's own tire mesh (24,836 nodes, 74,508 FEM
    dofs, 149,513 stored upper FEM blocks), plain FP64 Neumann order 2, omega 0.5."""
    s = tire_system
    assert s.layout[3] == 74508 and s.meta["tets"] == 78197
    fb0 = s.layout[2] // 3
    assert int(((s.rows >= fb0) & (s.cols >= fb0)).sum()) == 149513
    xo, so, orc = tire_oracle
    ctx = api.HSCContext(api.HSCOptions(neumann_order=2, omega=0.5, tol=1e-6))
    x, st = ctx.solve(api.DeviceSystem.from_system(s))
    assert st["status"] == 0
    assert st["rank"] == so["rank"]
    assert st["active_fem_dofs"] == so["active_fem_dofs"]
    k, a, act = ctx.factors()
    # the active FEM dofs, in the FEM block's own numbering, equal the oracle's extraction
    np.testing.assert_array_equal(np.sort(act), np.sort(orc.active))
    assert abs(st["pcg_iterations"] - so["pcg_iterations"]) <= 1
    assert rel(x.cpu().numpy(), xo) < 1e-5
    assert st["full_relative_residual"] <= 1e-6


def _errors(x, xr, H):
    e = x - xr
    return rel(x, xr), float(np.sqrt(abs(e @ (H @ e)) / abs(xr @ (H @ xr))))


@pytest.fixture(scope="module")
def tire_tight(api, tire_system):
    """FP64 solve of the tire-mesh system to a Schur residual of 1e-12: the reference solution
    the precision modes are measured against."""
    s = tire_system
    ref = api.HSCContext(api.HSCOptions(neumann_order=2, omega=0.5, tol=1e-12, max_iter=20000))
    xr, st = ref.solve(api.DeviceSystem.from_system(s))
    assert st["status"] == 0
    return xr.cpu().numpy()


@pytest.mark.parametrize("prec", ("fp32", "bf16"))
def test_tire_mesh_mixed_precision_error_against_fp64(api, torch, tire_system, tire_tight, prec):
    """Reduced-precision bulk against a tight FP64 solve of the same system (Schur tol 1e-12).
    At a 1e-6 residual this system (cond ~1e13) leaves a relative error of ~0.1 in x even in
    FP64, so the bar is the FP64 form's own error at the same tolerance: a precision mode may
    not be more than 2x (relative) / 2x (energy norm) farther from the tight solution."""
    s = tire_system
    ds = api.DeviceSystem.from_system(s)
    base = dict(neumann_order=2, omega=0.5, tol=1e-6, max_iter=20000)
    x64, _ = api.HSCContext(api.HSCOptions(**base)).solve(ds)
    r64, a64 = _errors(x64.cpu().numpy(), tire_tight, s.H)
    ctx = api.HSCContext(api.HSCOptions(precision=prec, residual_replacement=50, **base))
    x, st = ctx.solve(ds)
    assert st["status"] == 0 and st["full_relative_residual"] <= 1e-6
    r, a = _errors(x.cpu().numpy(), tire_tight, s.H)
    print(f"{prec}: rel {r:.3e} (fp64 {r64:.3e}), energy {a:.3e} (fp64 {a64:.3e})")
    assert r <= 2 * r64 + 1e-9, (r, r64)
    assert a <= 2 * a64 + 1e-9, (a, a64)


@pytest.mark.parametrize("prec", ("fp32", "bf16"))
def test_vehicle_mixed_precision_reaches_fp64_target(api, torch, vehicle_system, prec):
    """FP32 / BF16 bulk with FP64 residual replacement: the FP64 full residual
    still reaches 1e-6; the error against the FP64 direct solve is reported."""
    s = vehicle_system
    ctx = api.HSCContext(api.HSCOptions(neumann_order=2, tol=1e-6, precision=prec, residual_replacement=50,
                                        max_iter=20000))
    x, st = ctx.solve(api.DeviceSystem.from_system(s))
    assert st["status"] == 0
    assert st["full_relative_residual"] <= 1e-6


def test_solve_is_bitwise_deterministic(api, torch, vehicle_system):
    s = vehicle_system
    ctx = api.HSCContext(api.HSCOptions(neumann_order=2, tol=1e-6))
    ds = api.DeviceSystem.from_system(s)
    x1, st1 = ctx.solve(ds)
    x1 = x1.clone()
    x2, st2 = ctx.solve(ds)
    assert torch.equal(x1, x2)
    assert st1["pcg_iterations"] == st2["pcg_iterations"]


# ---------------------------------------------------------------------------
# batch, graph replay, edge cases and error paths
# ---------------------------------------------------------------------------
def test_batch_matches_single_solves(api, torch, golden, cube_system):
    systems_ = [fixture_system(golden, t) for t in STIFF] + [cube_system]
    opt = api.HSCOptions(max_rank=128, neumann_order=3, omega=2 / 3, tol=1e-9, full_residual_limit=1.0)
    ctx = api.HSCContext(opt)
    dss = [api.DeviceSystem.from_system(s) for s in systems_]
    xs, sts = ctx.solve_batch(dss)
    for s, ds, x, st in zip(systems_, dss, xs, sts):
        c1 = api.HSCContext(opt)
        x1, st1 = c1.solve(ds)
        assert st["status"] == 0
        assert abs(st["pcg_iterations"] - st1["pcg_iterations"]) <= 1
        assert rel(x.cpu().numpy(), x1.cpu().numpy()) < 1e-6


def test_batch_graph_replay(api, torch, golden, cube_system):
    systems_ = [fixture_system(golden, t) for t in STIFF] + [cube_system]
    opt = api.HSCOptions(max_rank=128, neumann_order=3, omega=2 / 3, tol=1e-9, full_residual_limit=1.0)
    ctx = api.HSCContext(opt)
    dss = [api.DeviceSystem.from_system(s) for s in systems_]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        xs = [torch.empty_like(d.b) for d in dss]
        xs, sts0 = ctx.solve_batch(dss, xs=xs, use_graph=True, stream=stream)
        ref = [x.clone() for x in xs]
        for d in dss:  # new right-hand sides behind the same pointers
            d.b.mul_(2.0)
        xs, sts1 = ctx.solve_batch(dss, xs=xs, use_graph=True, stream=stream)
    stream.synchronize()
    for x0, x1, a, b in zip(ref, xs, sts0, sts1):
        assert a["status"] == 0 and b["status"] == 0
        assert rel(x1.cpu().numpy(), 2.0 * x0.cpu().numpy()) < 1e-8


def test_zero_rhs_gives_zero(api, torch, cube_system):
    ctx = api.HSCContext(api.HSCOptions(omega=2 / 3))
    ds = api.DeviceSystem.from_system(cube_system)
    x, st = ctx.solve(ds, b=torch.zeros_like(ds.b), raise_on_error=False)
    assert st["pcg_iterations"] == 0
    assert torch.count_nonzero(x).item() == 0


def test_nonpositive_fem_diagonal_is_reported(api, torch, cube_system):
    s = cube_system
    ds = api.DeviceSystem.from_system(s)
    vals = ds.values.clone()
    rows, cols = s.rows, s.cols
    fb0 = s.layout[2] // 3
    k = int(np.flatnonzero((rows == cols) & (rows >= fb0))[5])
    vals[k] = -vals[k]
    bad = api.DeviceSystem(ds.rows, ds.cols, vals, ds.nblock, ds.layout, ds.b)
    ctx = api.HSCContext(api.HSCOptions(omega=2 / 3))
    x, st = ctx.solve(bad, raise_on_error=False)
    assert st["status"] == 2  # HSC_ERR_NONSPD


@pytest.mark.parametrize("drop", [False, True])
def test_uncoupled_system_solves_with_rank_zero(api, torch, cube_system, drop):
    """No ABD-FEM coupling (linear_hsc.cu:216-247 finds no active dof: every
    cross block is zero, or absent): rank 0, dq = A^-1 b_q, and the PCG over D
    alone meets the residual target.  (x itself is not compared with a direct
    solve: cond(D) of this cube is about 8e10.)"""
    s = cube_system
    qo, qm, fo, fn = s.layout
    qb = (s.rows < (qo + qm) // 3) != (s.cols < (qo + qm) // 3)
    assert qb.any()
    rows, cols, vals = s.rows, s.cols, s.vals.copy()
    if drop:
        rows, cols, vals = rows[~qb], cols[~qb], vals[~qb]
    else:
        vals[qb] = 0.0
    H = O.full_from_bcoo(rows, cols, vals, s.nblock)
    assert O.extract(H, s.layout)[3].size == 0
    cm = lambda v: torch.from_numpy(np.ascontiguousarray(np.transpose(v, (0, 2, 1)).reshape(-1, 9))).cuda()
    ds = api.DeviceSystem(torch.from_numpy(rows.astype(np.int32)).cuda(), torch.from_numpy(cols.astype(np.int32)).cuda(),
                          cm(vals), s.nblock, tuple(s.layout), torch.from_numpy(s.b).cuda())
    ctx = api.HSCContext(api.HSCOptions(omega=2 / 3, abd_inverse="exact"))
    x, st = ctx.solve(ds, raise_on_error=False)
    assert st["status"] == 0, st
    assert st["rank"] == 0 and st["active_fem_dofs"] == 0
    xh = x.cpu().numpy()
    A = H[qo:qo + qm, qo:qo + qm].toarray()
    assert rel(xh[qo:qo + qm], np.linalg.solve(A, s.b[qo:qo + qm])) <= 1e-8
    true_res = np.linalg.norm(H @ xh - s.b) / np.linalg.norm(s.b)
    assert st["full_relative_residual"] <= 1e-5 and true_res <= 1e-5, (st, true_res)


def test_iteration_cap_reports_noconv(api, torch, vehicle_system):
    ctx = api.HSCContext(api.HSCOptions(max_iter=5, tol=1e-12))
    x, st = ctx.solve(api.DeviceSystem.from_system(vehicle_system), raise_on_error=False)
    assert st["status"] == 4 and st["pcg_iterations"] == 5


def permuted(s, seed=1):
    """The same system with its FEM nodes renumbered: same nnzb, new pattern."""
    import scipy.sparse as sp
    qo, qm, fo, fn = s.layout
    rng = np.random.default_rng(seed)
    pi = rng.permutation(fn // 3)
    perm = np.arange(s.N)
    perm[fo:fo + fn] = fo + (3 * pi[:, None] + np.arange(3)).ravel()
    Pm = sp.csr_matrix((np.ones(s.N), (np.arange(s.N), perm)), shape=(s.N, s.N))
    H2 = (Pm @ s.H @ Pm.T).tocsr()
    rows, cols, vals = S.bcoo_upper_from_csr(H2)
    return S.HSCSystem("perm", s.layout, H2, rows, cols, vals, Pm @ s.b, Pm @ s.x_star, dict(s.meta))


def test_pattern_change_behind_same_pointers_is_reanalysed(api, torch, cube_system):
    """The analysis cache keys on pointers; a different pattern written into
    the same buffers is caught by the device-side pattern hash and analysed again."""
    s1 = cube_system
    s2 = permuted(s1)
    assert s2.rows.size == s1.rows.size and not np.array_equal(s2.cols, s1.cols)
    ctx = api.HSCContext(api.HSCOptions(omega=2 / 3, max_rank=128))
    ds = api.DeviceSystem.from_system(s1)
    x1, st1 = ctx.solve(ds)
    ds.rows.copy_(torch.from_numpy(s2.rows))
    ds.cols.copy_(torch.from_numpy(s2.cols))
    ds.values.copy_(torch.from_numpy(s2.values_colmajor()))
    ds.b.copy_(torch.from_numpy(s2.b))
    x2, st2 = ctx.solve(ds)
    xo, so, _ = O.hsc_solve(s2.H, s2.layout, s2.b, order=2, omega=2 / 3, tol=1e-6, max_iter=20000,
                            abd_inverse="exact", max_rank=128)
    assert abs(st2["pcg_iterations"] - so["pcg_iterations"]) <= 1
    assert rel(x2.cpu().numpy(), xo) < 1e-5


def test_refinement_reaches_target(api, torch, cube_system):
    """Quadratic refinement (core.py:171-198) over order-3 Neumann ABD-inverse
    directions: one direction leaves ~3.5e-7, refinement reaches 1e-9 in the
    same number of steps as the oracle."""
    s = cube_system
    opt = dict(neumann_order=3, omega=2 / 3, tol=1e-6, abd_inverse="neumann")
    ctx = api.HSCContext(api.HSCOptions(refine_target=1e-9, max_refinements=60, **opt))
    x, st = ctx.solve(api.DeviceSystem.from_system(s))
    xo, so, _ = O.hsc_solve(s.H, s.layout, s.b, order=3, omega=2 / 3, tol=1e-6, abd_inverse="neumann",
                            refine_target=1e-9, max_refinements=60)
    assert st["status"] == 0, st
    assert st["full_relative_residual"] <= 1e-9
    assert abs(st["refinement_steps"] - so["refinement_steps"]) <= 1
    # the FP64 residual of the returned x, recomputed on the CPU
    xs = x.cpu().numpy()
    assert np.linalg.norm(s.H @ xs - s.b) <= 1.01e-9 * np.linalg.norm(s.b)


def test_plugin_mirror_do_solve(api, torch, cube_system, tmp_path):
    plug = api.LinearHSC(workspace=str(tmp_path))
    plug.do_build({"linear_system/solver": "linear_hsc", "linear_system/tol_rate": 1e-6,
                   "linear_system/hsc/neumann_order": 2, "linear_system/hsc/omega": 2 / 3,
                   "linear_system/hsc/adaptive_abd_inverse": 1})
    ds = api.DeviceSystem.from_system(cube_system)
    info = api.SolvingInfo(ds)
    st = plug.do_solve(info)
    assert st["status"] == 0 and info.iter_count() == st["pcg_iterations"]
    import json
    rec = json.loads(open(tmp_path / "hsc_stats.jsonl").read().splitlines()[-1])
    for key in ("frame", "newton", "fem_dofs", "abd_dofs", "active_fem_dofs", "rank", "aca_relative_error",
                "pcg_iterations", "schur_relative_residual", "full_relative_residual", "setup_ms", "total_ms",
                "adaptive_abd_inverse", "neumann_doublings", "abd_inverse_residual", "full_residual_limit",
                "accepted", "solver", "fallback"):
        assert key in rec
    assert rec["solver"] == "linear_hsc" and rec["fallback"] is False and rec["accepted"] is True
