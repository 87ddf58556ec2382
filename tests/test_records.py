"""Solve evidence: the hsc_stats.jsonl collector (storage.py:17-62 semantics) and
the system dump / replay tool."""
import json

import numpy as np
import pytest

from hsc_reimpl_b200 import records as R


def _row(**kw):
    r = {"frame": 0, "newton": 0, "fem_dofs": 30, "abd_dofs": 12, "active_fem_dofs": 6, "rank": 4,
         "aca_relative_error": 1e-9, "pcg_iterations": 10, "schur_relative_residual": 5e-7,
         "full_relative_residual": 6e-7, "setup_ms": 1.0, "total_ms": 2.0, "active_mesh_contacts": 3,
         "active_ground_contacts": 2, "adaptive_abd_inverse": True, "neumann_doublings": 2,
         "abd_inverse_residual": 1e-6, "full_residual_limit": 0.1, "accepted": True,
         "solver": "linear_hsc", "fallback": False}
    r.update(kw)
    return json.dumps(r) + "\n"


def test_collector_copies_each_record_once_and_summarises(tmp_path):
    native, dest = tmp_path / "hsc_stats.jsonl", tmp_path / "copy.jsonl"
    rec = R.SolverRecords(native, dest)
    assert rec.collect() == []                     # no native log yet
    lines = [_row(rank=4, pcg_iterations=10, neumann_doublings=2),
             _row(newton=1, rank=9, pcg_iterations=7, full_relative_residual=2e-6, active_ground_contacts=5,
                  neumann_doublings=1)]
    native.write_text(lines[0] + lines[1][:20])    # the second record is still being written
    assert len(rec.collect()) == 1
    with native.open("a") as f:
        f.write(lines[1][20:])
    got = rec.collect()
    assert len(got) == 1 and got[0]["newton"] == 1
    assert rec.collect() == []                     # nothing new: nothing copied twice
    assert dest.read_text() == "".join(lines)
    s = rec.summary
    assert s["linear_solves"] == 2 and s["fallbacks"] == 0
    assert s["max_rank"] == 9 and s["min_rank"] == 4
    assert s["max_pcg_iterations"] == 10 and s["max_full_relative_residual"] == 2e-6
    assert s["max_ground_contacts"] == 5 and s["max_mesh_contacts"] == 3
    assert s["min_neumann_doublings"] == 1 and s["max_neumann_doublings"] == 2


@pytest.mark.parametrize("bad", [dict(fallback=True), dict(accepted=False), dict(solver="fused_pcg")])
def test_collector_rejects_unaccepted_solves(tmp_path, bad):
    native, dest = tmp_path / "hsc_stats.jsonl", tmp_path / "copy.jsonl"
    native.write_text(_row() + _row(newton=1, **bad))
    rec = R.SolverRecords(native, dest)
    with pytest.raises(R.UnacceptedSolve):
        rec.collect()
    assert rec.summary["linear_solves"] == 2


def test_dump_round_trip_on_host(tmp_path, cube_system):
    import torch
    from hsc_reimpl_b200.solver import DeviceSystem, HSCOptions
    s = cube_system
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    ds = DeviceSystem(t(s.rows.astype(np.int32)), t(s.cols.astype(np.int32)), t(s.values_colmajor()), s.nblock,
                      tuple(s.layout), t(s.b))
    opt = HSCOptions(precision="fp32", max_rank=64, poly_weights=(1.0, 0.5))
    x = torch.arange(s.N, dtype=torch.float64)
    R.dump_system(tmp_path / "s.npz", ds, options=opt, record={"pcg_iterations": 3}, x=x)
    ds2, o, rec, xr = R.load_system(tmp_path / "s.npz", device="cpu")
    for a in ("rows", "cols", "values", "b"):
        assert torch.equal(getattr(ds, a), getattr(ds2, a))
    assert ds2.nblock == ds.nblock and ds2.layout == ds.layout
    assert R.options_from_dict(o) == opt and rec == {"pcg_iterations": 3}
    assert np.array_equal(xr, x.numpy())
    assert R.options_from_dict(o, precision="fp64", max_rank=None).precision == "fp64"
    # a host HSCSystem dumps to the same arrays
    R.dump_system(tmp_path / "h.npz", s)
    ds3, _, _, _ = R.load_system(tmp_path / "h.npz", device="cpu")
    assert torch.equal(ds3.values, ds.values)


@pytest.mark.gpu
def test_replay_reproduces_dumped_solves(tmp_path, cube_system, vehicle_system):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200 import solver as api
    plug = api.LinearHSC(workspace=str(tmp_path), dump_systems=True)
    plug.do_build({"linear_system/solver": "linear_hsc", "linear_system/tol_rate": 1e-6,
                   "linear_system/hsc/omega": 2 / 3, "linear_system/hsc/adaptive_abd_inverse": 1})
    for k, s in enumerate((cube_system, vehicle_system)):
        plug.newton = k
        plug.do_solve(api.SolvingInfo(api.DeviceSystem.from_system(s)))
    rec = R.SolverRecords(tmp_path / "hsc_stats.jsonl", tmp_path / "copy.jsonl")
    assert len(rec.collect()) == 2
    rows = R.replay([str(tmp_path)])
    assert len(rows) == 2
    for r in rows:   # the solve is deterministic: same options, same bits
        assert r["accepted"] and r["pcg_iterations"] == r["recorded_pcg_iterations"]
        assert r["rank"] == r["recorded_rank"] and r["x_bitwise_equal"], r
    # with overrides: FP32 PCG with residual replacement, accepted with a full residual near the FP64
    # one's (the residual, not x, is the verified quantity: the cube's cond(H) is about 2e13)
    rows = R.replay([str(tmp_path)], precision="fp32", residual_replacement=50)
    for r in rows:
        assert r["accepted"] and not r["x_bitwise_equal"], r
        assert r["full_relative_residual"] <= max(10 * r["recorded_full_relative_residual"], 1e-5), r
