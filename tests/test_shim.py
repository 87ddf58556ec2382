"""The C++ LinearHSC plugin shim (hsc_reimpl_b200/shim/linear_hsc_shim.cpp),
compiled against the minimal libuipc mock and linked to libhsc_b200.so.

CPU: the plugin opts out with SimSystemException unless
linear_system/solver == "linear_hsc" (reference linear_hsc.cu:172-176) and
rejects invalid parameters with UIPC_ASSERT (:186-190).
GPU: one do_solve through the shim gives the same x, iteration count and
hsc_stats.jsonl record as the Python mirror of the plugin."""
import json
import subprocess

import numpy as np
import pytest

from hsc_reimpl_b200.shim import build_shim

CONFIG = {"linear_system/solver": "linear_hsc", "linear_system/tol_rate": 1e-6,
          "linear_system/hsc/neumann_order": 2, "linear_system/hsc/omega": 2 / 3,
          "linear_system/hsc/adaptive_abd_inverse": 1}


@pytest.fixture(scope="module")
def driver():
    try:
        return build_shim.build()
    except (RuntimeError, FileNotFoundError) as e:
        pytest.skip(f"shim driver not buildable here: {e}")


def run(driver, ws, system="-", config=CONFIG):
    args = [str(driver), str(ws), str(system)] + [f"{k}={v!r}" if not isinstance(v, str) else f"{k}={v}"
                                                   for k, v in config.items()]
    return subprocess.run(args, capture_output=True, text=True, timeout=600)


def write_system(path, s):
    qo, qm, fo, fn = s.layout
    with open(path, "wb") as f:
        f.write(np.int64(len(s.rows)).tobytes())
        f.write(np.array([s.nblock, qo, qm, fo, fn], np.int32).tobytes())
        f.write(np.ascontiguousarray(s.rows, np.int32).tobytes())
        f.write(np.ascontiguousarray(s.cols, np.int32).tobytes())
        f.write(s.values_colmajor().astype(np.float64).tobytes())
        f.write(np.ascontiguousarray(s.b, np.float64).tobytes())


def test_other_solver_opts_out(driver, tmp_path):
    r = run(driver, tmp_path, config={"linear_system/solver": "fused_pcg"})
    assert r.returncode == 2 and "LinearHSC unused" in r.stdout
    r = run(driver, tmp_path, config={})
    assert r.returncode == 2


@pytest.mark.parametrize("key,value", [("linear_system/hsc/omega", 1.5), ("linear_system/hsc/omega", 0.0),
                                       ("linear_system/hsc/max_rank", 0), ("linear_system/hsc/max_iter", -1),
                                       ("linear_system/hsc/neumann_order", 0)])
def test_invalid_parameters_assert(driver, tmp_path, key, value):
    r = run(driver, tmp_path, config={**CONFIG, key: value})
    assert r.returncode == 3 and "Invalid HSC parameters" in r.stdout


@pytest.mark.gpu
def test_shim_solve_matches_python_plugin(driver, tmp_path, cube_system):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200 import solver as api
    sysfile = tmp_path / "cube.bin"
    write_system(sysfile, cube_system)
    (tmp_path / "shim").mkdir()
    r = run(driver, tmp_path / "shim", sysfile)
    assert r.returncode == 0, r.stdout + r.stderr
    x_shim = np.fromfile(tmp_path / "shim" / "x.bin", np.float64)
    rec = json.loads((tmp_path / "shim" / "hsc_stats.jsonl").read_text().splitlines()[-1])

    (tmp_path / "py").mkdir()
    plug = api.LinearHSC(workspace=str(tmp_path / "py"))
    plug.do_build(CONFIG)
    info = api.SolvingInfo(api.DeviceSystem.from_system(cube_system))
    st = plug.do_solve(info)
    x_py = info.x().cpu().numpy()
    ref = json.loads((tmp_path / "py" / "hsc_stats.jsonl").read_text().splitlines()[-1])

    assert f"iterations {st['pcg_iterations']}" in r.stdout
    assert np.array_equal(x_shim, x_py)  # same library, same options: bitwise
    assert set(ref) <= set(rec)
    for k in ("pcg_iterations", "rank", "fem_dofs", "abd_dofs", "active_fem_dofs", "accepted", "solver",
              "fallback", "adaptive_abd_inverse", "neumann_doublings"):
        assert rec[k] == ref[k], k
    assert rec["full_relative_residual"] == pytest.approx(ref["full_relative_residual"], rel=1e-12)
    assert np.linalg.norm(cube_system.H @ x_shim - cube_system.b) <= 1e-5 * np.linalg.norm(cube_system.b)


@pytest.mark.gpu
def test_shim_record_counts_active_contacts(driver, tmp_path, cube_system):
    """The record's active contact counts come from the scene's trajectory filters as in the
    reference (linear_hsc.cu:410-414): PT + EE + PE + PP simplex pairs, PH vertex-half-plane pairs;
    a scene without a filter reports 0 for it."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sysfile = tmp_path / "cube.bin"
    write_system(sysfile, cube_system)
    cases = [({"contacts/PT": 3, "contacts/EE": 2, "contacts/PE": 1, "contacts/PP": 4, "contacts/PH": 5}, 10, 5),
             ({"contacts/PH": 7}, 0, 7), ({}, 0, 0)]
    for i, (contacts, mesh, ground) in enumerate(cases):
        ws = tmp_path / f"ws{i}"
        ws.mkdir()
        r = run(driver, ws, sysfile, config={**CONFIG, **contacts})
        assert r.returncode == 0, r.stdout + r.stderr
        rec = json.loads((ws / "hsc_stats.jsonl").read_text().splitlines()[-1])
        assert rec["active_mesh_contacts"] == mesh and rec["active_ground_contacts"] == ground, rec
