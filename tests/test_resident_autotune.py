"""The shared-memory-resident PCG path (each CTA keeps its BSR slice, vector
window and own-row vectors in shared memory) against the streaming path, and
the batch autotuner, which keeps a candidate only if every system meets the
FP64-verified residual target."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16"])
def test_resident_and_streaming_agree(api, torch, vehicle_system, prec):
    """The resident kernel (BSR slice, vector window and own-row vectors in
    shared memory, four threads per row) and the streaming one (warp segmented
    scan over L2) sum each row in a different order, so they agree to the
    solve's accuracy, with the same iteration count within one; every tile
    width of one path gives the same answer to that accuracy too."""
    ds = api.DeviceSystem.from_system(vehicle_system)
    rr = 0 if prec == "fp64" else 50
    s = vehicle_system
    outs = {}
    for tpr in (2, 4, 8):
        for resident in (False, True):
            ctx = api.HSCContext(api.HSCOptions(precision=prec, residual_replacement=rr, resident=resident,
                                                threads_per_row=tpr))
            x, st = ctx.solve(ds)
            outs[(resident, tpr)] = (x.cpu().numpy(), st["pcg_iterations"])
    ref, it0 = outs[(False, 4)]
    for (resident, tpr), (x, it) in outs.items():
        assert abs(it - it0) <= 2, (resident, tpr, it, it0)
        assert np.linalg.norm(x - ref) <= 1e-5 * np.linalg.norm(ref)
        assert np.linalg.norm(s.H @ x - s.b) <= 1.01e-6 * np.linalg.norm(s.b)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fused_update_agrees_with_separate_phases(api, torch, vehicle_system, prec):
    """Resident mode with the update folded into the first preconditioner
    phase (one grid barrier fewer) against the separate-phase schedule."""
    ds = api.DeviceSystem.from_system(vehicle_system)
    rr = 0 if prec == "fp64" else 50
    out = []
    for fuse in (False, True):
        ctx = api.HSCContext(api.HSCOptions(precision=prec, residual_replacement=rr, resident=True, fuse_update=fuse))
        x, st = ctx.solve(ds)
        out.append((x.cpu().numpy(), st["pcg_iterations"], st["full_relative_residual"]))
    assert abs(out[0][1] - out[1][1]) <= 2
    assert np.linalg.norm(out[0][0] - out[1][0]) <= 1e-5 * np.linalg.norm(out[0][0])
    assert out[1][2] <= 1e-6


def test_resident_is_deterministic(api, torch, vehicle_system):
    ds = api.DeviceSystem.from_system(vehicle_system)
    ctx = api.HSCContext(api.HSCOptions(resident=True))
    x1, _ = ctx.solve(ds)
    x1 = x1.cpu().numpy()
    x2, _ = api.HSCContext(api.HSCOptions(resident=True)).solve(ds)
    assert np.array_equal(x1, x2.cpu().numpy())


def test_resident_schur_polynomial_matches_streaming(api, torch, vehicle_system):
    ds = api.DeviceSystem.from_system(vehicle_system)
    res = []
    for resident in (False, True):
        ctx = api.HSCContext(api.HSCOptions(poly_weights=(1.0,) * 8, poly_basis="schur", resident=resident))
        x, st = ctx.solve(ds)
        res.append((x.cpu().numpy(), st["pcg_iterations"]))
    assert abs(res[0][1] - res[1][1]) <= 2
    assert np.linalg.norm(res[0][0] - res[1][0]) <= 1e-5 * np.linalg.norm(res[0][0])


def test_autotuner_picks_a_candidate_that_meets_the_target(api, torch):
    from hsc_reimpl_b200 import autotune
    from hsc_reimpl_b200.systems import make_cube_system, make_torus_system
    systems = [make_cube_system(seed=1, n=6, h=0.1 / 6, E=1e7),
               make_torus_system(seed=2, target_tets=3000, bodies=3, E=1e8),
               make_torus_system(seed=3, target_tets=5000, bodies=5, E=1e6)]
    # rank caps 16 and 64: the oracle breaks down below the coupling rank (31 and 55 here) and
    # converges at 64, so the tuner must reject every rank-16 candidate
    best, table = autotune.autotune(systems, tiles=(2, 4), ranks=(16, 64), reps=2)
    assert len(table) == 4
    assert best is not None, table
    ok = [r for r in table if r["ok"]]
    assert all(r["max_full_relative_residual"] <= 1e-6 for r in ok)
    assert all(r["max_rank"] == 64 for r in ok) and len(ok) == 2, table
    fastest = min(ok, key=lambda r: r["ms"])
    assert (best.threads_per_row, best.max_rank) == (fastest["threads_per_row"], fastest["max_rank"])


@pytest.mark.parametrize("resident", [False, True])
def test_partition_weights_agree(api, torch, vehicle_system, monkeypatch, resident):
    """The CTA row partition weights each coupled node by its low-rank work; the weight moves row
    boundaries and so the reduction order only: every weight gives the same solve to its tolerance."""
    ds = api.DeviceSystem.from_system(vehicle_system)
    outs = {}
    for w in ("0", "0.5", "2", "8"):
        monkeypatch.setenv("HSC_ACTIVE_ROW_WEIGHT", w)
        ctx = api.HSCContext(api.HSCOptions(resident=resident))
        x, st = ctx.solve(ds)
        assert st["status"] == 0 and st["full_relative_residual"] <= 1e-6, (w, st)
        outs[w] = (x.cpu().numpy(), st["pcg_iterations"])
        ctx.close()
    x0, it0 = outs["0"]
    for w, (x, it) in outs.items():
        assert abs(it - it0) <= 2, (w, it, it0)
        assert np.linalg.norm(x - x0) <= 1e-5 * np.linalg.norm(x0), w
