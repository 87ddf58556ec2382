"""The shared-memory-resident SpMV path (each CTA keeps its BSR slice and
vector window in shared memory) and the SpMV tile width change where data
come from, not the arithmetic: results are bit-identical to the streaming
path.  The batch autotuner keeps a candidate only if every system meets the
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
def test_resident_and_tile_width_are_bit_identical(api, torch, vehicle_system, prec):
    ds = api.DeviceSystem.from_system(vehicle_system)
    rr = 0 if prec == "fp64" else 50
    outs = []
    for resident, tpr in ((False, 4), (True, 4), (True, 2), (True, 8)):
        ctx = api.HSCContext(api.HSCOptions(precision=prec, residual_replacement=rr, resident=resident,
                                            threads_per_row=tpr))
        x, st = ctx.solve(ds)
        outs.append((x.cpu().numpy(), st["pcg_iterations"]))
    for x, it in outs[1:]:
        assert it == outs[0][1]
        assert np.array_equal(x, outs[0][0])


def test_resident_schur_polynomial_matches_streaming(api, torch, vehicle_system):
    ds = api.DeviceSystem.from_system(vehicle_system)
    res = []
    for resident in (False, True):
        ctx = api.HSCContext(api.HSCOptions(poly_weights=(1.0,) * 8, poly_basis="schur", resident=resident))
        x, st = ctx.solve(ds)
        res.append((x.cpu().numpy(), st["pcg_iterations"]))
    assert res[0][1] == res[1][1] and np.array_equal(res[0][0], res[1][0])


def test_autotuner_picks_a_candidate_that_meets_the_target(api, torch):
    from hsc_reimpl_b200 import autotune
    from hsc_reimpl_b200.systems import make_cube_system, make_torus_system
    systems = [make_cube_system(seed=1, n=6, h=0.1 / 6, E=1e7),
               make_torus_system(seed=2, target_tets=3000, bodies=3, E=1e8),
               make_torus_system(seed=3, target_tets=5000, bodies=5, E=1e6)]
    best, table = autotune.autotune(systems, tiles=(2, 4), ranks=(4, 32), reps=2)
    assert len(table) == 4
    assert best is not None
    ok = [r for r in table if r["ok"]]
    assert all(r["max_full_relative_residual"] <= 1e-6 for r in ok)
    fastest = min(ok, key=lambda r: r["ms"])
    assert (best.threads_per_row, best.max_rank) == (fastest["threads_per_row"], fastest["max_rank"])
