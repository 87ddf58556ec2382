"""Generate the golden vectors in this folder from the reference's own NumPy core.

Run in a container where the reference checkout exists (it is read, never
written):

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py <reference-checkout> [--only projection]

It imports ``reproduction/core.py`` unmodified and records:

* ``manufactured.npz`` -- ``core.manufactured_system`` for stiffness
  1e2/1e4/1e6 (checked equal to the reference's saved
  ``reproduction/results/fixture_*.npz``) and, per stiffness and Neumann order
  1/3/5/8, the ``HSC(...).solve`` solution and iteration count (checked equal
  to ``reproduction/results/summary.csv``), the ACA factors and history and
  the affine Neumann inverse;
* ``checks.npz`` -- the inputs and outputs of the 13 numerical checks of
  ``reproduction/run.py:70-107``;
* ``cube.npz`` -- ``core.HSC`` on the 1,331-node cube system made by
  ``hsc_reimpl_b200.systems.make_cube_system(seed=0)`` at order 2, omega 2/3,
  ACA rtol 1e-4, PCG rtol 1e-6 (one solve, the exact-affine variant and
  ``core.refinement`` to a 1e-6 full residual).  Only outputs and an input
  checksum are stored; the inputs are regenerated from the seed;
* ``projection.npz`` -- ``core.affine_projection`` (``core.py:201-206``), the
  3x12 affine-body Jacobian of the reference's core, at 64 seeded rest points
  (numpy ``default_rng(206)``, standard normal, the first one the origin).
"""
import csv
import hashlib
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def input_digest(H, b):
    h = hashlib.sha256()
    Hc = H.tocsr()
    Hc.sort_indices()
    for a in (Hc.indptr, Hc.indices, Hc.data, b):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def projection(core):
    rest = np.random.default_rng(206).standard_normal((64, 3))
    rest[0] = 0.0
    P = np.stack([core.affine_projection(r) for r in rest])
    np.savez_compressed(HERE / "projection.npz", rest=rest, P=P)


def main(ref_root, only=None):
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(Path(ref_root) / "reproduction"))
    import core  # the reference's NumPy HSC core, unmodified

    if only in (None, "projection"):
        projection(core)
    if only == "projection":
        return

    out = {}
    saved_summary = {}
    with open(Path(ref_root) / "reproduction/results/summary.csv", encoding="utf-8-sig") as f:
        for row in csv.DictReader(f):
            saved_summary[(float(row["stiffness"]), int(row["order"]))] = int(row["inner_iterations"])
    for stiffness in (1e2, 1e4, 1e6):
        tag = f"{stiffness:.0e}"
        D, A, E, H, b, x_star = core.manufactured_system(stiffness)
        saved = np.load(Path(ref_root) / f"reproduction/results/fixture_{tag}.npz")
        assert np.max(np.abs(saved["D"] - D)) < 1e-9 * np.max(np.abs(D))
        assert np.max(np.abs(saved["b"] - b)) < 1e-12
        out[f"{tag}/D"], out[f"{tag}/A"], out[f"{tag}/E"], out[f"{tag}/b"] = D, A, E, b
        out[f"{tag}/x_direct"] = saved["x_direct"]
        n, m = len(D), len(A)
        for order in (1, 3, 5, 8):
            solver = core.HSC(D, A, E, order=order, omega=0.7, aca_max_rank=min(m, n))
            x, info = solver.solve(b)
            assert info["iterations"] == saved_summary[(stiffness, order)], (stiffness, order, info)
            out[f"{tag}/o{order}/x"] = x
            out[f"{tag}/o{order}/iterations"] = np.int64(info["iterations"])
            out[f"{tag}/o{order}/history"] = np.asarray(info["history"])
            out[f"{tag}/o{order}/P"] = solver.affine_neumann(np.eye(m))
            out[f"{tag}/o{order}/C"] = solver.C
        f = core.aca(E, max_rank=min(m, n))
        out[f"{tag}/aca/U"], out[f"{tag}/aca/V"] = f.U, f.V
        out[f"{tag}/aca/residuals"] = np.asarray(f.residuals)
        out[f"{tag}/aca/pivots"] = np.asarray([p[:2] for p in f.pivots], dtype=np.int64)
        ex = core.HSC(D, A, E, exact_affine=True)
        x, info = ex.solve(b)
        out[f"{tag}/exact/x"] = x
        out[f"{tag}/exact/iterations"] = np.int64(info["iterations"])
    np.savez_compressed(HERE / "manufactured.npz", **out)

    # the numerical checks of run.py:70-107, inputs and outputs
    chk = {}
    rng = np.random.default_rng(501)
    U, V = rng.normal(size=(24, 4)), rng.normal(size=(45, 4))
    E = U @ V.T
    f = core.aca(E, rtol=1e-12)
    chk["aca_E"], chk["aca_U"], chk["aca_V"] = E, f.U, f.V
    chk["aca_rank"] = np.int64(f.rank)
    chk["aca_fixed3_rank"] = np.int64(core.aca(E, max_rank=3).rank)
    A = rng.normal(size=(24, 24))
    A = A.T @ A + 50 * np.eye(24)
    op = core.Neumann(A, 12, 5, 0.7)
    chk["neumann_A"], chk["neumann_M"] = A, op(np.eye(24))
    D, A2, E2, H, b, _ = core.manufactured_system(stiffness=1e4, nx=4, ny=2, nz=2)
    solver = core.HSC(D, A2, E2, exact_affine=True)
    x, info = solver.solve(b, rtol=1e-12)
    chk["small_D"], chk["small_A"], chk["small_E"], chk["small_b"] = D, A2, E2, b
    chk["small_x"] = x
    chk["small_iterations"] = np.int64(info["iterations"])
    direction = rng.normal(size=len(D))
    chk["small_direction"] = direction
    chk["small_schur_mv"] = solver.matvec(direction)
    np.savez_compressed(HERE / "checks.npz", **chk)

    # the 1,331-node cube system, order 2, ACA rtol 1e-4, PCG 1e-6.  At nu=0.45
    # lambda_max(B^-1 D) is 2.91 > 2/0.7, so the order-2 Neumann polynomial with
    # omega=0.7 is indefinite there; omega=2/3 is the authors' own default
    # (Guo-2026-HSC conjugate_gradient_cuda.cuh:115).
    from hsc_reimpl_b200.systems import make_cube_system
    s = make_cube_system(seed=0)
    qo, qm, fo, fn = s.layout
    Hd = s.H.toarray()
    D, A, E = Hd[fo:fo + fn, fo:fo + fn], Hd[qo:qo + qm, qo:qo + qm], Hd[qo:qo + qm, fo:fo + fn]
    # core.py orders FEM first, ABD last
    b_core = np.concatenate([s.b[fo:fo + fn], s.b[qo:qo + qm]])
    cube = {"digest": np.frombuffer(input_digest(s.H, s.b).encode(), dtype=np.uint8)}
    solver = core.HSC(D, A, E, order=2, omega=2/3, aca_rtol=1e-4)
    x, info = solver.solve(b_core, rtol=1e-6, maxiter=20000)
    cube["o2/x"] = x
    cube["o2/iterations"] = np.int64(info["iterations"])
    cube["o2/rank"] = np.int64(solver.factors.rank)
    cube["o2/aca_residuals"] = np.asarray(solver.factors.residuals)
    Hcore = np.block([[D, E.T], [E, A]])
    cube["o2/full_residual"] = np.float64(np.linalg.norm(Hcore @ x - b_core) / np.linalg.norm(b_core))
    ex = core.HSC(D, A, E, order=2, omega=2/3, aca_rtol=1e-4, exact_affine=True)
    x, info = ex.solve(b_core, rtol=1e-6, maxiter=20000)
    cube["exact/x"] = x
    cube["exact/iterations"] = np.int64(info["iterations"])
    cube["exact/full_residual"] = np.float64(np.linalg.norm(Hcore @ x - b_core) / np.linalg.norm(b_core))
    xr, outer = core.refinement(Hcore, b_core, ex, rtol=1e-6)
    cube["refine/x"] = xr
    cube["refine/steps"] = np.int64(outer["steps"])
    cube["refine/inner"] = np.asarray(outer["inner_iterations"], dtype=np.int64)
    cube["refine/history"] = np.asarray(outer["history"])
    np.savez_compressed(HERE / "cube.npz", **cube)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    if only:
        args = [a for a in args if a != only]
    main(args[0] if args else "/root/reference", only)
