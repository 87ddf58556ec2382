"""GPU assembly of the log-Neo-Hookean FEM Hessian (hsc_fem_assemble) against
the NumPy restatement of the reference's per-tet Hessian and assembly, and a
solve of a device-assembled system through the same C ABI."""
import numpy as np
import pytest

from oracle import fem_oracle as F
from oracle import hsc_oracle as O
from hsc_reimpl_b200 import systems as S


def test_oracle_assembly_matches_the_generator():
    """The oracle's assembly equals the system generator's (an independent
    NumPy path: COO triplets, scipy CSR, upper blocks) on a perturbed cube."""
    rng = np.random.default_rng(3)
    x, tets = S.cube_mesh(4, 0.05)
    h = np.cbrt((np.abs(np.linalg.det(x[tets[:, 1:]] - x[tets[:, :1]])) / 6.0).mean())  # as the generator
    xp = x + 0.02 * h * rng.standard_normal(x.shape)
    rows, cols, vals = F.assemble(tets, x, xp, 1e6, nu=0.45)
    r, c, v, _ = S.fem_hessian(x, tets, 1e6, 0.45, 1000.0, perturb=0.02, rng=np.random.default_rng(3))
    import scipy.sparse as sp
    H = sp.coo_matrix((v, (r, c)), shape=(3 * len(x),) * 2).tocsr()
    rr, cc, vv = S.bcoo_upper_from_csr(H)
    assert np.array_equal(rows, rr) and np.array_equal(cols, cc)
    vv = np.transpose(vv, (0, 2, 1)).reshape(-1, 9)
    assert np.max(np.abs(vals - vv)) <= 1e-9 * np.max(np.abs(vv))


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("mesh", ["cube", "tire"])
def test_gpu_assembly_matches_oracle(torch, mesh):
    from hsc_reimpl_b200.assembly import FemAssembler
    rng = np.random.default_rng(7)
    if mesh == "cube":
        x, tets = S.cube_mesh(10, 0.01)
        nu, E = 0.45, 1e6 * np.exp(rng.uniform(-1, 1, len(tets)))
    else:
        x, tets, _ = S.annulus_mesh()
        nu, E = 0.3, 1e8 * np.exp(rng.uniform(-1, 1, len(tets)))
    h = np.cbrt(np.abs(np.linalg.det(x[tets[:, 1:]] - x[tets[:, :1]])).mean() / 6)
    xp = x + 0.02 * h * rng.standard_normal(x.shape)
    asm = FemAssembler(tets, x, rho=1000.0, nu=nu)
    vals = asm.assemble(xp, E).cpu().numpy()
    rows, cols, ref = F.assemble(tets, x, xp, E, nu=nu)
    assert np.array_equal(asm.rows.cpu().numpy(), rows) and np.array_equal(asm.cols.cpu().numpy(), cols)
    # Jacobi (device) and LAPACK (oracle) eigen-decompositions agree to roundoff of the projection
    err = np.max(np.abs(vals - ref), axis=1) / np.max(np.abs(ref), axis=1)
    assert err.max() <= 1e-9, err.max()
    # the assembly is deterministic
    again = asm.assemble(xp, E).cpu().numpy()
    assert np.array_equal(vals, again)


@pytest.mark.gpu
def test_inverted_tet_is_reported(torch):
    from hsc_reimpl_b200.assembly import FemAssembler
    from hsc_reimpl_b200._lib import HSCError
    x, tets = S.cube_mesh(3, 0.1)
    asm = FemAssembler(tets, x)
    xp = x.copy()
    xp[tets[0, 1]] = xp[tets[0, 0]] - (xp[tets[0, 1]] - xp[tets[0, 0]]) * 2.0  # flip one corner through
    with pytest.raises(HSCError, match="nonspd"):
        asm.assemble(xp, 1e6)


@pytest.mark.gpu
def test_device_assembled_system_solves(torch):
    """FEM block assembled on the device, plus an affine plate touching the
    bottom face (host-built here), solved through hsc_solve: x matches the
    oracle's solve of the same matrix."""
    from hsc_reimpl_b200.assembly import FemAssembler
    from hsc_reimpl_b200 import solver as api
    rng = np.random.default_rng(11)
    n_cell, hh = 6, 0.02
    x, tets = S.cube_mesh(n_cell, hh)
    xp = x + 0.02 * hh * rng.standard_normal(x.shape)
    nn = len(x)
    asm = FemAssembler(tets, x, nu=0.45)
    fem_vals = asm.assemble(xp, 1e6)
    # ABD plate (12 dofs first) with stitches to the bottom nodes, assembled on the host
    qm = 12
    A = S._Assembler(qm + 3 * nn)
    bottom = np.flatnonzero(np.isclose(x[:, 2], 0.0))
    c0 = np.array([n_cell * hh / 2, n_cell * hh / 2, -hh])
    A.add_dense(np.arange(12), S.abd_block(50.0, x[bottom] - c0, 1e10, (n_cell * hh) ** 2 * hh))
    for node in bottom:
        S._stitch(A, qm, node, 0, x[node] - c0, 1e7)
    Hc = A.csr()
    cr, cc, cv = S.bcoo_upper_from_csr(Hc)                 # ABD + coupling + contact diagonal parts
    fr = asm.rows.cpu().numpy() + qm // 3
    fc = asm.cols.cpu().numpy() + qm // 3
    keys_f = fr.astype(np.int64) * (qm // 3 + nn) + fc
    keys_c = cr.astype(np.int64) * (qm // 3 + nn) + cc
    allk = np.unique(np.concatenate([keys_f, keys_c]))
    pos_f = np.searchsorted(allk, keys_f)
    pos_c = np.searchsorted(allk, keys_c)
    vals = torch.zeros(len(allk), 9, dtype=torch.float64, device="cuda")
    vals.index_add_(0, torch.from_numpy(pos_f).cuda(), fem_vals)                # device-assembled block, no host copy
    vals.index_add_(0, torch.from_numpy(pos_c).cuda(),
                    torch.from_numpy(np.transpose(cv, (0, 2, 1)).reshape(-1, 9).copy()).cuda())
    nb = qm // 3 + nn
    rows = torch.from_numpy((allk // nb).astype(np.int32)).cuda()
    cols = torch.from_numpy((allk % nb).astype(np.int32)).cuda()
    H = O.full_from_bcoo(rows.cpu().numpy(), cols.cpu().numpy(),
                         np.transpose(vals.cpu().numpy().reshape(-1, 3, 3), (0, 2, 1)), nb)
    b = H @ rng.standard_normal(3 * nb)
    layout = (0, qm, qm, 3 * nn)
    ds = api.DeviceSystem(rows, cols, vals, nb, layout, torch.from_numpy(b).cuda())
    opts = dict(neumann_order=2, omega=2 / 3, tol=1e-8, abd_inverse="exact")
    xg, st = api.HSCContext(api.HSCOptions(**opts)).solve(ds)
    xo, so, _ = O.hsc_solve(H, layout, b, order=2, omega=2 / 3, tol=1e-8, abd_inverse="exact", max_iter=20000,
                            max_rank=128)
    assert abs(st["pcg_iterations"] - so["pcg_iterations"]) <= 1
    assert np.linalg.norm(xg.cpu().numpy() - xo) <= 1e-6 * np.linalg.norm(xo)
    assert st["full_relative_residual"] <= 1e-7


def test_oracle_feasibility_rule():
    """A segment that passes through an inverted state between two positive
    endpoints is infeasible (the reason for checking the derivative roots)."""
    A = np.eye(3)
    E = np.diag([1.0, 1.0, 1.0])
    E[2, 2] = 1.0
    assert F.segment_feasible(A, E)
    # det(A + s B) = (1 - 2 s)^2 (1 + ...) dips to 0 at s = 0.5 while both ends are positive
    A = np.diag([1.0, 1.0, 1.0])
    E = np.diag([-1.0, -1.0, 1.0])
    assert np.linalg.det(E) > 0
    assert not F.segment_feasible(A, E)


@pytest.mark.gpu
@pytest.mark.parametrize("scale", [0.05, 0.6, 3.0])
def test_gpu_feasible_step_matches_oracle(torch, scale):
    from hsc_reimpl_b200.assembly import FemAssembler
    rng = np.random.default_rng(int(scale * 100))
    x, tets = S.cube_mesh(5, 0.02)
    dx = scale * 0.02 * rng.standard_normal(x.shape)
    asm = FemAssembler(tets, x)
    got = asm.feasible_step(x, dx, alpha0=1.0, max_halvings=40)
    ref = F.feasible_step(tets, x, x, dx, alpha0=1.0, max_halvings=40)
    assert got[1] == ref[1] and got[2] == ref[2]
    assert got[0] == ref[0]
    if scale < 0.1:
        assert got == (1.0, 0, 0)
    else:
        assert got[1] > 0


def test_oracle_feasible_step_is_tight():
    """The returned step keeps every tet feasible and twice it does not."""
    rng = np.random.default_rng(3)
    x, tets = S.cube_mesh(2, 0.02)
    dx = 0.04 * rng.standard_normal(x.shape)
    alpha, m, lim = F.feasible_step(tets, x, x, dx, alpha0=1.0, max_halvings=40)
    assert m > 0 and lim > 0 and alpha == 2.0 ** -m
    a1, m1, _ = F.feasible_step(tets, x, x, alpha * dx, alpha0=1.0, max_halvings=40)
    assert (a1, m1) == (1.0, 0)
    _, m2, _ = F.feasible_step(tets, x, x, 2 * alpha * dx, alpha0=1.0, max_halvings=40)
    assert m2 == 1


@pytest.mark.gpu
def test_gpu_feasible_step_rejects_inverted_start(torch):
    from hsc_reimpl_b200.assembly import FemAssembler
    x, tets = S.cube_mesh(3, 0.02)
    asm = FemAssembler(tets, x)
    xi = x.copy()
    xi[:, 2] *= -1.0  # mirrored: every tet inverted at s = 0
    alpha, m, lim = asm.feasible_step(xi, np.zeros_like(x), alpha0=1.0, max_halvings=8)
    assert alpha == 0.0 and m == 9 and lim == len(tets)
    assert F.feasible_step(tets, x, xi, np.zeros_like(x), 1.0, 8) == (0.0, 9, len(tets))
    # a half step along a feasible direction
    alpha, m, lim = asm.feasible_step(x, np.zeros_like(x), alpha0=0.5, max_halvings=8)
    assert (alpha, m, lim) == (0.5, 0, 0)


# The reference's native segment checks (reproduction/hsc_backend/check_log_nh.cpp:78-87):
# (end matrix, feasible from the identity)
def _segment_cases():
    two_roots = np.eye(3); two_roots[0, 0] = -3; two_roots[1, 1] = -1     # det < 0 between 1/4 and 1/2
    double_root = np.eye(3); double_root[0, 0] = -1; double_root[1, 1] = -1  # det touches 0 at 1/2
    inverted_end = np.eye(3); inverted_end[2, 2] = -0.1
    return [(two_roots, False), (double_root, False), (inverted_end, False), (0.25 * np.eye(3), True),
            (np.eye(3), True)]


def test_oracle_segment_known_answers():
    for E, ok in _segment_cases():
        assert F.segment_feasible(np.eye(3), E) == ok


@pytest.mark.gpu
def test_gpu_segment_known_answers(torch):
    """One unit tet (Dm = I, so F = Ds): the step from the rest shape to F = E."""
    from hsc_reimpl_b200.assembly import FemAssembler
    rest = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
    tets = np.array([[0, 1, 2, 3]], dtype=np.int32)
    asm = FemAssembler(tets, rest)
    for E, ok in _segment_cases():
        end = np.vstack([np.zeros(3), E.T])  # node k = column k of F
        got = asm.feasible_step(rest, end - rest, alpha0=1.0, max_halvings=0)
        assert got == ((1.0, 0, 0) if ok else (0.0, 1, 1)), (E, got)
