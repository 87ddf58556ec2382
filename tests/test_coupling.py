"""ABD-FEM contact coupling assembled on the device, fused with the active-column
and E extraction (hsc_coupling.cu), against the NumPy oracle
(oracle/coupling_oracle.py) and, through a solve, against a direct solve."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import coupling_oracle as CO
from oracle import hsc_oracle as O
from hsc_reimpl_b200 import systems as S

PERM_LIB = np.r_[9:12, 0:9]   # libuipc order (p, a1, a2, a3) from the core order (a1, a2, a3, p)


def scene(seed, nbody=5, nv_per_body=40, nfem=300, ncontact=2500, fixed=True):
    rng = np.random.default_rng(seed)
    v2b = np.repeat(np.arange(nbody), nv_per_body).astype(np.int32)
    xbar = rng.uniform(-1, 1, (len(v2b), 3))
    # few distinct (body, node) pairs, so many contacts share a pair
    av = rng.integers(0, len(v2b), ncontact).astype(np.int32)
    fv = rng.integers(0, nfem // 3, ncontact).astype(np.int32) * 3 + rng.integers(0, 2, ncontact).astype(np.int32)
    n = rng.standard_normal((ncontact, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    k = rng.uniform(0.5, 2.0, ncontact)
    H = -(k[:, None, None] * n[:, :, None] * n[:, None, :])      # the (ABD vertex, FEM node) block of k n n^T
    H[rng.random(ncontact) < 0.05] = 0.0                         # contacts with a zero Hessian
    body_fixed = np.zeros(nbody, np.int32)
    fem_fixed = np.zeros(nfem, np.int32)
    if fixed:
        body_fixed[nbody - 1] = 1                                # e.g. the ground
        fem_fixed[rng.choice(nfem, 10, replace=False)] = 1
    return dict(v2b=v2b, xbar=xbar, av=av, fv=fv, H=H, k=k, n=n, body_fixed=body_fixed, fem_fixed=fem_fixed,
                nbody=nbody, nfem=nfem)


def colmajor(H):
    return np.ascontiguousarray(np.transpose(H, (0, 2, 1)).reshape(-1, 9))


# ----------------------------------------------------------------------------- CPU
def test_oracle_jacobian_orders():
    xb = np.array([0.3, -1.2, 2.0])
    assert np.array_equal(CO.jacobian(xb, p_first=False), S.affine_projection(xb))
    assert np.array_equal(CO.jacobian(xb, p_first=True), S.affine_projection(xb)[:, PERM_LIB])
    q = np.random.default_rng(0).standard_normal(12)       # x = p + A xbar
    A, p = q[3:].reshape(3, 3), q[:3]
    assert np.allclose(CO.jacobian(xb) @ q, p + A @ xb)


def test_oracle_fused_extraction_matches_extraction_from_the_global_matrix():
    """E and the active dofs built from the pairs equal what the solver's setup
    extracts from the assembled global matrix (hsc_oracle.extract)."""
    sc = scene(1)
    nbody, nfem = sc["nbody"], sc["nfem"]
    pairs = CO.coupling_blocks(sc["v2b"], sc["xbar"], sc["av"], sc["fv"], sc["H"], sc["body_fixed"], sc["fem_fixed"])
    rows, cols, vals = CO.bcoo(pairs, 0, 4 * nbody)
    nblock = 4 * nbody + nfem
    diag = np.arange(nblock)
    allr = np.concatenate([rows, diag]); allc = np.concatenate([cols, diag])
    allv = np.concatenate([vals, np.repeat(np.eye(3)[None], nblock, 0)])
    Hg = O.full_from_bcoo(allr, allc, allv, nblock)
    layout = (0, 12 * nbody, 12 * nbody, 3 * nfem)
    _, _, E_ref, act_ref = O.extract(Hg, layout)
    act, E = CO.extract(pairs, nbody, 4 * nbody)
    assert np.array_equal(act, act_ref + 12 * nbody)
    assert np.array_equal(E, E_ref)
    assert act.size and act.size < 3 * nfem                  # fixed nodes / zero contacts drop out


# ----------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def device_and_oracle(sc, p_first, fem_off=None):
    from hsc_reimpl_b200.assembly import CouplingAssembler
    fem_off = 4 * sc["nbody"] if fem_off is None else fem_off
    ca = CouplingAssembler(sc["v2b"], sc["xbar"], sc["nbody"], sc["nfem"], sc["body_fixed"], sc["fem_fixed"],
                           abd_block_offset=0, fem_block_offset=fem_off, p_first=p_first)
    got = ca.assemble(sc["av"], sc["fv"], colmajor(sc["H"]))
    pairs = CO.coupling_blocks(sc["v2b"], sc["xbar"], sc["av"], sc["fv"], sc["H"], sc["body_fixed"],
                               sc["fem_fixed"], p_first=p_first)
    return ca, got, pairs


@pytest.mark.gpu
@pytest.mark.parametrize("p_first", [True, False])
@pytest.mark.parametrize("seed", [0, 1])
def test_gpu_coupling_matches_oracle_bitwise(torch, p_first, seed):
    sc = scene(seed)
    ca, got, pairs = device_and_oracle(sc, p_first)
    rows, cols, vals = CO.bcoo(pairs, 0, 4 * sc["nbody"])
    act, E = CO.extract(pairs, sc["nbody"], 4 * sc["nbody"])
    assert np.array_equal(got["rows"].cpu().numpy(), rows)
    assert np.array_equal(got["cols"].cpu().numpy(), cols)
    assert np.array_equal(got["values"].cpu().numpy(), colmajor(vals))
    assert np.array_equal(got["active"].cpu().numpy(), act)
    assert np.array_equal(got["E"].cpu().numpy(), E)
    again = ca.assemble(sc["av"], sc["fv"], colmajor(sc["H"]))       # repeat: same bits
    for key in got:
        assert torch.equal(got[key], again[key])
    # contacts in another order: the same blocks up to the summation order
    perm = np.random.default_rng(5).permutation(len(sc["av"]))
    sh = ca.assemble(sc["av"][perm], sc["fv"][perm], colmajor(sc["H"][perm]))
    assert torch.equal(sh["rows"], got["rows"]) and torch.equal(sh["active"], got["active"])
    assert torch.allclose(sh["values"], got["values"], rtol=1e-13, atol=1e-13)


@pytest.mark.gpu
def test_gpu_coupling_edge_cases(torch):
    from hsc_reimpl_b200._lib import HSCError
    sc = scene(2, fixed=False)
    ca, got, pairs = device_and_oracle(sc, True)
    assert got["E"].shape[1] == got["active"].numel() > 0
    empty = ca.assemble(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 9)))
    assert empty["rows"].numel() == 0 and empty["E"].shape == (12 * sc["nbody"], 0)
    bad = sc["fv"].copy()
    bad[7] = sc["nfem"]                                       # node out of range
    with pytest.raises(HSCError):
        ca.assemble(sc["av"], bad, colmajor(sc["H"]))
    # every body fixed: no blocks, no active dofs
    sc2 = dict(sc, body_fixed=np.ones(sc["nbody"], np.int32))
    _, g2, _ = device_and_oracle(sc2, True)
    assert g2["rows"].numel() == 0 and g2["active"].numel() == 0


@pytest.mark.gpu
def test_gpu_coupled_system_solves(torch):
    """FEM block + ABD blocks + the device-assembled coupling, solved by HSC."""
    from hsc_reimpl_b200.solver import DeviceSystem, HSCContext, HSCOptions
    rng = np.random.default_rng(3)
    x, tets, _ = S.annulus_mesh(nr=2, na=3, nc=24)
    nfem, nbody = len(x), 3
    fr, fc, fvv, node_mass = S.fem_hessian(x, tets, 1e6, 0.3, 1000.0)
    nv = 30
    v2b = np.repeat(np.arange(nbody), nv).astype(np.int32)
    xbar = rng.uniform(-0.5, 0.5, (len(v2b), 3))
    nc = 400
    av = rng.integers(0, len(v2b), nc).astype(np.int32)
    fv = rng.integers(0, nfem, nc).astype(np.int32)
    nrm = rng.standard_normal((nc, 3)); nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    K = 1e3 * rng.uniform(0.5, 2, nc)[:, None, None] * nrm[:, :, None] * nrm[:, None, :]
    qm, N = 12 * nbody, 12 * nbody + 3 * nfem
    # ABD blocks (libuipc order): dyadic mass + the contacts' J^T K J; FEM diagonal: + K
    Hd = sp.lil_matrix((N, N))
    for b in range(nbody):
        M = S.abd_block(50.0, xbar[v2b == b], 1e7, 1e-2)[np.ix_(PERM_LIB, PERM_LIB)]
        Hd[12 * b:12 * b + 12, 12 * b:12 * b + 12] = M
    Hd = Hd.tocsr() + sp.csr_matrix((fvv, (fr + qm, fc + qm)), shape=(N, N))
    add = sp.lil_matrix((N, N))
    for t in range(nc):
        b, f = v2b[av[t]], fv[t]
        J = CO.jacobian(xbar[av[t]])
        add[12 * b:12 * b + 12, 12 * b:12 * b + 12] += J.T @ K[t] @ J
        add[qm + 3 * f:qm + 3 * f + 3, qm + 3 * f:qm + 3 * f + 3] += K[t]
    Hd = (Hd + add.tocsr()).tocsr()
    Hd = ((Hd + Hd.T) * 0.5).tocsr()
    r0, c0, v0 = S.bcoo_upper_from_csr(Hd)
    from hsc_reimpl_b200.assembly import CouplingAssembler
    ca = CouplingAssembler(v2b, xbar, nbody, nfem, fem_block_offset=4 * nbody)
    cp = ca.assemble(av, fv, colmajor(-K))
    rows = torch.cat([torch.from_numpy(r0).cuda(), cp["rows"]])
    cols = torch.cat([torch.from_numpy(c0).cuda(), cp["cols"]])
    vals = torch.cat([torch.from_numpy(np.ascontiguousarray(np.transpose(v0, (0, 2, 1)).reshape(-1, 9))).cuda(),
                      cp["values"]])
    Hfull = O.full_from_bcoo(rows.cpu().numpy(), cols.cpu().numpy(),
                             np.transpose(vals.cpu().numpy().reshape(-1, 3, 3), (0, 2, 1)), N // 3)
    assert np.all(np.linalg.eigvalsh(Hfull.toarray()) > 0)
    b = rng.standard_normal(N)
    ds = DeviceSystem(rows.contiguous(), cols.contiguous(), vals.contiguous(), N // 3, (0, qm, qm, 3 * nfem),
                      torch.from_numpy(b).cuda())
    ctx = HSCContext(HSCOptions(tol=1e-10, max_rank=qm, omega=0.6))
    xs, st = ctx.solve(ds, raise_on_error=False)
    assert st["status"] == 0, st
    assert st["active_fem_dofs"] == cp["active"].numel()
    xref = sp.linalg.spsolve(Hfull.tocsc(), b)
    assert np.linalg.norm(xs.cpu().numpy() - xref) <= 1e-6 * np.linalg.norm(xref)
    # the solver's own coupling factors see the same active dofs the assembler returned
    _, _, _, act = O.extract(Hfull, (0, qm, qm, 3 * nfem))
    assert np.array_equal(cp["active"].cpu().numpy(), act + qm)
