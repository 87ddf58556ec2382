"""CPU oracle for one HSC linear solve.  TEST INFRASTRUCTURE ONLY.

This module is the checker: only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline legs of ``bench.py`` may import it.  The product path
(``hsc_reimpl_b200``) never calls it.

It restates, in NumPy/SciPy, the reference's algorithm for the path:

* ``aca``           -- full-pivot ACA, ``reproduction/core.py:22-50``
                       (row-major first-occurrence argmax, ``eps*max(scale,tiny)``
                       zero-pivot guard, optional Frobenius ``rtol``);
* ``block_inverse`` -- block-Jacobi inverse with an SPD check, ``core.py:53-71``;
* ``neumann_dense`` -- the Neumann polynomial ``sum_k T^k w B^-1``,
                       ``core.py:74-88``; the adaptive doubling
                       ``P <- P + P(I - A P)`` of ``linear_hsc.cu:276-297``;
* ``extract``       -- DOF split, dense A / E over sorted active FEM dofs,
                       ``linear_hsc.cu:195-247``;
* ``pcg_schur``     -- the Schur PCG loop with a recursive-residual test and
                       one true-residual check on convergence,
                       ``linear_hsc.cu:359-393`` (``core.py:95-138`` tests the
                       true residual each iteration instead);
* ``hsc_solve``     -- ``linear_hsc.cu:344-406`` / ``core.py:141-168`` plus the
                       quadratic refinement of ``core.py:171-198``;
* ``direct_solve``  -- the FP64 direct-solve oracle (``scipy.sparse.linalg.splu``);
* ``hsc_solve_block`` -- this build's fast form (no reference counterpart): the
                       block-local polynomial preconditioner with the exact Woodbury
                       correction for the coupling, in a pipelined PCG; its setup is
                       the reference's (``core.py:141-168``).

Parity pins: ``tests/golden`` holds outputs of the reference's own
``core.py`` (generated by ``tests/golden/make_golden.py``); the CPU tests
check this restatement against them.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

EPS = np.finfo(np.float64).eps
TINY = np.finfo(np.float64).tiny


# ----------------------------------------------------------------------------
# input form
# ----------------------------------------------------------------------------
def full_from_bcoo(rows, cols, vals, nblock):
    """Full symmetric CSR from one stored triangle of 3x3 blocks.

    An off-diagonal block (i, j, B) stands for B at (i, j) and B^T at (j, i);
    a diagonal block is stored once (``linear_hsc.cu:59-60``,
    ``spmv.cu:631-660``).  ``vals`` is (nnzb, 3, 3) row-major.
    """
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64).reshape(-1, 3, 3)
    off = rows != cols
    r = np.concatenate([rows, cols[off]])
    c = np.concatenate([cols, rows[off]])
    v = np.concatenate([vals, np.transpose(vals[off], (0, 2, 1))])
    ii = (3 * r[:, None, None] + np.arange(3)[None, :, None]).repeat(3, 2)
    jj = (3 * c[:, None, None] + np.arange(3)[None, None, :]).repeat(3, 1)
    N = 3 * nblock
    return sp.coo_matrix((v.ravel(), (ii.ravel(), jj.ravel())), shape=(N, N)).tocsr()


def extract(H, layout):
    """Split H into D (sparse FEM block), dense A, dense E (qm x a) and the
    sorted active FEM dofs (columns of a nonzero coupling 3x3 block).

    ``linear_hsc.cu:216-247``: a FEM node is active when any of its coupling
    blocks has a nonzero squared norm; all three of its dofs become columns.
    """
    qo, qm, fo, fn = layout
    H = sp.csr_matrix(H)
    D = H[fo:fo + fn, fo:fo + fn].tocsr()
    A = H[qo:qo + qm, qo:qo + qm].toarray()
    Ef = H[qo:qo + qm, fo:fo + fn].tocsc()
    nz = np.zeros(fn // 3, dtype=bool)
    Ef.eliminate_zeros()
    colnz = np.diff(Ef.indptr) > 0
    nz[:] = colnz.reshape(-1, 3).any(1)
    nodes = np.flatnonzero(nz)
    active = (3 * nodes[:, None] + np.arange(3)).ravel()
    E = Ef[:, active].toarray() if active.size else np.zeros((qm, 0))
    return D, A, E, active


# ----------------------------------------------------------------------------
# ACA
# ----------------------------------------------------------------------------
def aca(E, rtol=None, max_rank=None):
    """Full-pivot ACA, ``core.py:22-50``.  Returns (U, V, residuals, pivots)."""
    E = np.asarray(E, dtype=np.float64)
    if E.ndim != 2 or not np.isfinite(E).all() or (rtol is not None and rtol < 0):
        raise ValueError("ACA requires a finite matrix and nonnegative tolerance")
    m, n = E.shape
    limit = min(m, n) if max_rank is None else min(max_rank, m, n)
    R = E.copy()
    scale = np.linalg.norm(E)
    residuals, pivots, us, vs = [1.0 if scale else 0.0], [], [], []
    while len(us) < limit and residuals[-1] > (0.0 if rtol is None else rtol):
        flat = int(np.argmax(np.abs(R)))
        i, j = divmod(flat, n)
        pivot = R[i, j]
        if abs(pivot) <= EPS * max(scale, TINY):
            break
        u = R[:, j].copy()
        v = R[i, :].copy() / pivot
        us.append(u)
        vs.append(v)
        pivots.append((i, j, float(pivot)))
        R -= np.outer(u, v)
        residuals.append(float(np.linalg.norm(R) / scale))
    U = np.column_stack(us) if us else np.zeros((m, 0))
    V = np.column_stack(vs) if vs else np.zeros((n, 0))
    return U, V, residuals, pivots


# ----------------------------------------------------------------------------
# block inverses and Neumann polynomials
# ----------------------------------------------------------------------------
def block_inverse(M, bs):
    """Inverses of the bs x bs diagonal blocks; raises on a non-SPD block
    (``core.py:53-71``, ``linear_hsc.cu:264-271``)."""
    n = M.shape[0]
    if n % bs:
        raise ValueError("block size must divide the matrix")
    out = np.empty((n // bs, bs, bs))
    for k in range(n // bs):
        s = slice(k * bs, (k + 1) * bs)
        blk = np.asarray(M[s, s].toarray() if sp.issparse(M) else M[s, s], dtype=np.float64)
        np.linalg.cholesky(blk)
        out[k] = np.linalg.solve(blk, np.eye(bs))
    return out


def block_diag_apply(inv, r):
    bs = inv.shape[1]
    return np.einsum("kij,kj->ki", inv, r.reshape(-1, bs)).ravel()


def fem_diag_inverse(D):
    """3x3 diagonal-block inverses of the FEM block; ``linear_hsc.cu:70-80``
    rejects a block whose determinant is not positive and finite."""
    n = D.shape[0] // 3
    Db = sp.csr_matrix(D).tobsr(blocksize=(3, 3))
    Db.sort_indices()
    blocks = np.zeros((n, 3, 3))
    for i in range(n):
        lo, hi = Db.indptr[i], Db.indptr[i + 1]
        k = np.searchsorted(Db.indices[lo:hi], i)
        if k < hi - lo and Db.indices[lo + k] == i:
            blocks[i] = Db.data[lo + k]
    det = np.linalg.det(blocks)
    bad = ~(np.isfinite(det) & (det > 0))
    if bad.any():
        raise np.linalg.LinAlgError(f"{int(bad.sum())} non-positive FEM diagonal blocks")
    return np.linalg.inv(blocks)


def neumann_weights(order, weights=None):
    w = np.ones(order) if weights is None else np.asarray(weights, dtype=np.float64)
    if w.size < 1:
        raise ValueError("empty polynomial")
    return w


def neumann_apply(D, Dinv, r, order=5, omega=0.7, weights=None):
    """z = sum_k w_k t_k,  t_0 = w B^-1 r,  t_k = t_{k-1} - w B^-1 D t_{k-1}.

    With unit weights this is ``core.py:82-88`` / ``linear_hsc.cu:330-343``.
    """
    w = neumann_weights(order, weights)
    term = omega * block_diag_apply(Dinv, r)
    z = w[0] * term
    for k in range(1, w.size):
        term = term - omega * block_diag_apply(Dinv, D @ term)
        z = z + w[k] * term
    return z


def schur_poly_apply(schur, Dinv, r, order=5, omega=0.7, weights=None):
    """The Schur-basis polynomial of the learned preconditioner (no reference
    counterpart): the Neumann recursion of ``neumann_apply`` with the Schur
    operator S = D - V C V^T in place of D,
    z = sum_k w_k t_k,  t_0 = w B^-1 r,  t_k = t_{k-1} - w B^-1 S t_{k-1}."""
    w = neumann_weights(order, weights)
    term = omega * block_diag_apply(Dinv, r)
    z = w[0] * term
    for k in range(1, w.size):
        term = term - omega * block_diag_apply(Dinv, schur(term))
        z = z + w[k] * term
    return z


def neumann_dense(A, bs, order, omega):
    """Explicit P = sum_{k<order} T^k w B^-1 with T = I - w B^-1 A,
    symmetrised (``linear_hsc.cu:263-275``; ``core.py:74-88`` applied to I)."""
    inv = block_inverse(A, bs)
    n = A.shape[0]
    B = np.zeros((n, n))
    for k in range(n // bs):
        B[k * bs:(k + 1) * bs, k * bs:(k + 1) * bs] = inv[k]
    T = np.eye(n) - omega * B @ A
    term = omega * B
    P = term.copy()
    for _ in range(1, order):
        term = T @ term
        P += term
    return (P + P.T) * 0.5


def abd_inverse(A, mode="exact", order=5, omega=0.7, tol=1e-5, max_doublings=48):
    """ABD inverse approximation P.  Modes:

    * ``neumann``  -- fixed-order Neumann (``core.py:148``);
    * ``adaptive`` -- Neumann extended by doubling until
      ``|I - A P|_F / sqrt(qm) <= tol`` (``linear_hsc.cu:276-297``);
    * ``exact``    -- the dense FP64 inverse (``core.py:149-150``).
    Returns (P, doublings, inverse_residual).
    """
    qm = A.shape[0]
    if qm == 0:
        return np.zeros((0, 0)), 0, 0.0
    if mode == "exact":
        L = np.linalg.cholesky(A)
        Li = np.linalg.solve(L, np.eye(qm))
        P = Li.T @ Li
        P = (P + P.T) * 0.5
        return P, 0, float(np.linalg.norm(np.eye(qm) - A @ P) / np.sqrt(qm))
    P = neumann_dense(A, 12, order, omega)
    I = np.eye(qm)
    Rr = I - A @ P
    err = float(np.linalg.norm(Rr) / np.sqrt(qm))
    d = 0
    while mode == "adaptive" and err > tol and d < max_doublings:
        P = P + P @ Rr
        P = (P + P.T) * 0.5
        Rr = I - A @ P
        err = float(np.linalg.norm(Rr) / np.sqrt(qm))
        d += 1
        if not (np.isfinite(P).all() and np.isfinite(err)):
            raise ArithmeticError(f"ABD Neumann extension diverged at doubling {d}")
    if mode == "adaptive" and err > tol:
        raise ArithmeticError(f"ABD inverse residual {err} exceeds {tol} after {d} doublings")
    return P, d, err


# ----------------------------------------------------------------------------
# Schur PCG
# ----------------------------------------------------------------------------
class BreakdownError(ArithmeticError):
    pass


def pcg_schur(matvec, rhs, precond, tol, max_iter, history=None):
    """PCG with the recursive-residual stop test and one true-residual check
    at convergence (restart if it fails), ``linear_hsc.cu:359-393``."""
    x = np.zeros_like(rhs)
    r = rhs.copy()
    normb = float(np.linalg.norm(rhs))
    relative = 1.0 if normb > 0 else 0.0
    it = 0
    alphas, betas = [], []
    if normb > 0:
        z = precond(r)
        p = z.copy()
        rz = float(r @ z)
        while it < max_iter and relative > tol:
            Ap = matvec(p)
            denom = float(p @ Ap)
            if not (np.isfinite(denom) and denom > 0 and np.isfinite(rz) and rz > 0):
                raise BreakdownError(f"Schur PCG breakdown at iteration {it}: pSp={denom}, rz={rz}")
            alpha = rz / denom
            alphas.append(alpha)
            x += alpha * p
            r -= alpha * Ap
            it += 1
            relative = float(np.linalg.norm(r)) / normb
            if history is not None:
                history.append(relative)
            if relative <= tol:
                r = rhs - matvec(x)
                relative = float(np.linalg.norm(r)) / normb
                if relative <= tol:
                    break
                z = precond(r)
                p = z.copy()
                rz = float(r @ z)
                betas.append(0.0)
                continue
            z = precond(r)
            nxt = float(r @ z)
            beta = nxt / rz
            betas.append(beta)
            p = z + beta * p
            rz = nxt
    return x, dict(iterations=it, relative=relative, converged=relative <= tol,
                   alphas=alphas, betas=betas)


DEFAULTS = dict(max_rank=128, aca_rtol=None, order=5, omega=0.7, tol=1e-4, max_iter=2000,
                abd_inverse="adaptive", abd_inverse_tol=1e-5, weights=None, basis="fem",
                full_residual_limit=0.1, refine_target=None, max_refinements=20)


class HSCOracle:
    """Setup of one HSC system: ACA, ABD inverse, reduced core C = U^T P U."""

    def __init__(self, H, layout, **opts):
        o = dict(DEFAULTS)
        o.update(opts)
        self.o = o
        self.layout = layout
        self.H = sp.csr_matrix(H)
        qo, qm, fo, fn = layout
        if not (qm >= 0 and fn > 0 and qm % 12 == 0 and fn % 3 == 0 and qm + fn == self.H.shape[0]):
            raise ValueError("HSC requires only ABD (12/body) and FEM (3/node) dofs")
        self.D, self.A, self.E, self.active = extract(self.H, layout)
        self.Dinv = fem_diag_inverse(self.D)
        cap = min(o["max_rank"], qm, self.active.size)
        self.U, self.V, self.aca_hist, self.pivots = aca(self.E, rtol=o["aca_rtol"], max_rank=cap)
        self.rank = self.U.shape[1]
        self.aca_error = self.aca_hist[-1] if self.aca_hist else 0.0
        if qm:
            self.P, self.doublings, self.abd_err = abd_inverse(
                self.A, o["abd_inverse"], o["order"], o["omega"], o["abd_inverse_tol"])
        else:
            self.P, self.doublings, self.abd_err = np.zeros((0, 0)), 0, 0.0
        C = self.U.T @ self.P @ self.U
        self.C = (C + C.T) * 0.5

    def schur(self, p):
        y = self.D @ p
        if self.rank:
            t = self.V.T @ p[self.active]
            y[self.active] -= self.V @ (self.C @ t)
        return y

    def precond(self, r):
        o = self.o
        if o["basis"] == "schur":
            return schur_poly_apply(self.schur, self.Dinv, r, o["order"], o["omega"], o["weights"])
        return neumann_apply(self.D, self.Dinv, r, o["order"], o["omega"], o["weights"])

    def solve_once(self, b, history=None):
        """One HSC direction for right-hand side b (``linear_hsc.cu:344-406``)."""
        qo, qm, fo, fn = self.layout
        o = self.o
        bq, bx = b[qo:qo + qm], b[fo:fo + fn]
        rhs = bx.copy()
        if self.rank:
            c = self.U.T @ (self.P @ bq)
            rhs[self.active] -= self.V @ c
        dx, st = pcg_schur(self.schur, rhs, self.precond, o["tol"], o["max_iter"], history)
        if self.rank:
            vt = self.V.T @ dx[self.active]
            dq = self.P @ (bq - self.U @ vt)
        else:
            dq = self.P @ bq
        x = np.zeros_like(b)
        x[fo:fo + fn] = dx
        x[qo:qo + qm] = dq
        return x, st


def hsc_solve(H, layout, b, **opts):
    """Full HSC solve with stats; optional quadratic refinement to a full-system
    target (``core.py:171-198``).  Returns (x, stats)."""
    orc = HSCOracle(H, layout, **opts)
    o = orc.o
    b = np.asarray(b, dtype=np.float64)
    bn = float(np.linalg.norm(b))
    if o["refine_target"] is None or bn == 0:
        x, st = orc.solve_once(b)
        total_iters = st["iterations"]
        steps = 1
        full = float(np.linalg.norm(b - orc.H @ x) / bn) if bn > 0 else 0.0
        descent = float(b @ x)
    else:
        # the first direction is the first refinement step (x starts at 0, alpha
        # by exact line search as in core.py:186-191)
        x = np.zeros_like(b)
        r = b.copy()
        steps = 0
        total_iters = 0
        d, st = orc.solve_once(r)
        while True:
            total_iters += st["iterations"]
            steps += 1
            num = float(r @ d)
            Hd = orc.H @ d
            den = float(d @ Hd)
            if num <= 0 or den <= 0:
                raise ArithmeticError("approximate HSC direction is not descent")
            alpha = min(1.0, num / den)
            x += alpha * d
            r = b - orc.H @ x
            full = float(np.linalg.norm(r) / bn)
            if full <= o["refine_target"] or steps >= o["max_refinements"]:
                break
            d, st = orc.solve_once(r)
        descent = float(b @ x)
    stats = dict(fem_dofs=layout[3], abd_dofs=layout[1], active_fem_dofs=int(orc.active.size),
                 rank=orc.rank, aca_relative_error=orc.aca_error, pcg_iterations=total_iters,
                 last_pcg_iterations=st["iterations"], schur_relative_residual=st["relative"],
                 full_relative_residual=full, neumann_doublings=orc.doublings,
                 abd_inverse_residual=orc.abd_err, refinement_steps=steps, descent=descent,
                 converged=bool(st["converged"]))
    return x, stats, orc


def direct_solve(H, b):
    """FP64 direct solve of the full system (splu)."""
    lu = spla.splu(sp.csc_matrix(H))
    return lu.solve(np.asarray(b, dtype=np.float64))


# ----------------------------------------------------------------------------
# Block-local preconditioner with the exact coupling correction, pipelined PCG
# (this build's fast form; no reference counterpart -- the reference's
# preconditioner is the global Neumann series above)
# ----------------------------------------------------------------------------
def part_of_nodes(perm, part_ptr):
    """part id of every caller node from the solver's internal numbering (hsc_get_partition)."""
    perm = np.asarray(perm)
    out = np.empty(perm.size, dtype=np.int64)
    for p in range(len(part_ptr) - 1):
        out[perm[part_ptr[p]:part_ptr[p + 1]]] = p
    return out


def local_block(D, part, offdiag=False):
    """D with only the 3x3 blocks whose row and column nodes share a part (without the
    diagonal blocks when ``offdiag``)."""
    Db = sp.csr_matrix(D).tobsr(blocksize=(3, 3))
    Db.sort_indices()
    n = Db.shape[0] // 3
    rows = np.repeat(np.arange(n), np.diff(Db.indptr))
    keep = part[rows] == part[Db.indices]
    if offdiag:
        keep &= rows != Db.indices
    Dl = sp.bsr_matrix((Db.data * keep[:, None, None], Db.indices, Db.indptr), shape=D.shape).tocsr()
    Dl.eliminate_zeros()
    return Dl


def block_poly_apply(Ol, Dinv, r, weights, omega):
    """L r = sum_k w_k t_k, t_0 = w Dd^-1 r, t_k = t_{k-1} - w Dd^-1 D_loc t_{k-1}, evaluated as
    t_k = (1 - w) t_{k-1} - w Dd^-1 O_loc t_{k-1} with O_loc = D_loc minus its diagonal blocks
    (Dd^-1 D_loc = I + Dd^-1 O_loc), the order the CUDA kernel takes; r may hold columns."""
    def bd(v):
        if v.ndim == 1:
            return block_diag_apply(Dinv, v)
        n = Dinv.shape[0]
        return np.einsum("kij,kjc->kic", Dinv, v.reshape(n, 3, -1)).reshape(v.shape)
    term = omega * bd(r)
    z = weights[0] * term
    for k in range(1, len(weights)):
        term = (1.0 - omega) * term - omega * bd(Ol @ term)
        z = z + weights[k] * term
    return z


def ldlt(C):
    """C = L diag(d) L^T, L unit lower triangular (no pivoting)."""
    k = C.shape[0]
    L = np.eye(k)
    d = np.zeros(k)
    A = np.array(C, dtype=np.float64)
    for j in range(k):
        d[j] = A[j, j] - (L[j, :j] ** 2) @ d[:j]
        for i in range(j + 1, k):
            L[i, j] = (A[i, j] - (L[i, :j] * L[j, :j]) @ d[:j]) / d[j]
    return L, d


class BlockWoodbury:
    """z = L r + Y K Y^T r with L the block-local polynomial, Y = L V (V embedded at the
    active FEM dofs) and K = (C^-1 - V^T Y)^-1, formed as L_c (diag(1/d) - L_c^T G L_c)^-1 L_c^T
    from C = L_c diag(d) L_c^T, G = V^T Y.  With L = D^-1 this is S^-1 exactly (Woodbury), so
    the PCG iterates only against the error of the local polynomial.  Y is rounded to FP32, as
    the device applies it.  A failed Cholesky of K^-1 leaves z = L r."""

    def __init__(self, orc, part, weights, omega):
        self.Ol = local_block(orc.D, part, offdiag=True)
        self.Dinv = orc.Dinv
        self.w = np.asarray(weights, dtype=np.float64)
        self.omega = omega
        N = orc.D.shape[0]
        k = orc.rank
        self.K = np.zeros((k, k))
        self.Y = np.zeros((N, k))
        self.spd = True
        if k:
            Vf = np.zeros((N, k))
            Vf[orc.active] = orc.V
            self.Y = block_poly_apply(self.Ol, self.Dinv, Vf, self.w, omega).astype(np.float32).astype(np.float64)
            G = Vf.T @ self.Y
            G = 0.5 * (G + G.T)
            Lc, d = ldlt(orc.C)
            Ki = np.diag(1.0 / d) - Lc.T @ G @ Lc
            Ki = 0.5 * (Ki + Ki.T)
            try:
                Lk = np.linalg.cholesky(Ki)
                Kt = np.linalg.solve(Lk.T, np.linalg.solve(Lk, np.eye(k)))
                self.K = Lc @ Kt @ Lc.T
                self.K = 0.5 * (self.K + self.K.T)
            except np.linalg.LinAlgError:
                self.spd = False

    def __call__(self, r):
        z = block_poly_apply(self.Ol, self.Dinv, r, self.w, self.omega)
        if self.K.size:
            z = z + self.Y @ (self.K @ (self.Y.T @ r))
        return z


def pcg_pipelined(matvec, rhs, precond, tol, max_iter, rr_every=0):
    """Pipelined PCG (Ghysels & Vanroose 2014): one reduction phase per iteration overlaps the
    preconditioner and the operator product of the next.  Recursive-residual stop test, then one
    true-residual check; a failed check (or every ``rr_every`` iterations) restarts from the true
    residual.  Returns (x, stats)."""
    x = np.zeros_like(rhs)
    normb = float(np.linalg.norm(rhs))
    if normb == 0:
        return x, dict(iterations=0, relative=0.0, converged=True, restarts=0)
    r = rhs.copy()
    u = precond(r)
    w = matvec(u)
    z = q = s = p = np.zeros_like(rhs)
    it = restarts = 0
    alpha_prev = gamma_prev = None
    rel = 1.0
    while True:
        gamma, delta, rr = float(r @ u), float(w @ u), float(r @ r)
        rel = np.sqrt(rr) / normb
        replace = rr_every > 0 and it > 0 and it % rr_every == 0 and alpha_prev is not None
        if rel <= tol or replace or it >= max_iter:
            rt = rhs - matvec(x)
            rel = float(np.linalg.norm(rt)) / normb
            restarts += 1
            if rel <= tol or it >= max_iter:
                break
            r = rt
            u = precond(r)
            w = matvec(u)
            alpha_prev = None
            continue
        m = precond(w)
        nv = matvec(m)
        if alpha_prev is None:
            beta = 0.0
            den = delta
        else:
            beta = gamma / gamma_prev
            den = delta - beta * gamma / alpha_prev
        if not (np.isfinite(den) and den > 0 and np.isfinite(gamma) and gamma > 0):
            raise BreakdownError(f"pipelined PCG breakdown at iteration {it}: den={den}, gamma={gamma}")
        alpha = gamma / den
        z = nv + beta * z
        q = m + beta * q
        s = w + beta * s
        p = u + beta * p
        x = x + alpha * p
        r = r - alpha * s
        u = u - alpha * q
        w = w - alpha * z
        alpha_prev, gamma_prev = alpha, gamma
        it += 1
    return x, dict(iterations=it, relative=rel, converged=rel <= tol, restarts=restarts)


def hsc_solve_block(H, layout, b, perm, part_ptr, weights, omega, tol=1e-6, max_iter=20000, rr_every=0,
                    max_rank=128):
    """The fast form end to end: the reference's setup (ACA, exact ABD inverse, C = U^T P U,
    Schur rhs), the block-local Woodbury preconditioner over the solver's parts, pipelined PCG,
    back-substitution.  Returns (x, stats, oracle, preconditioner)."""
    orc = HSCOracle(H, layout, order=2, omega=omega, tol=tol, max_iter=max_iter, abd_inverse="exact",
                    max_rank=max_rank)
    qo, qm, fo, fn = layout
    part = part_of_nodes(perm, part_ptr)
    M = BlockWoodbury(orc, part, weights, omega)
    b = np.asarray(b, dtype=np.float64)
    bq, bx = b[qo:qo + qm], b[fo:fo + fn]
    rhs = bx.copy()
    if orc.rank:
        c = orc.U.T @ (orc.P @ bq)
        rhs[orc.active] -= orc.V @ c
    dx, st = pcg_pipelined(orc.schur, rhs, M, tol, max_iter, rr_every)
    if orc.rank:
        dq = orc.P @ (bq - orc.U @ (orc.V.T @ dx[orc.active]))
    else:
        dq = orc.P @ bq
    x = np.zeros_like(b)
    x[fo:fo + fn] = dx
    x[qo:qo + qm] = dq
    bn = float(np.linalg.norm(b))
    st = dict(st, pcg_iterations=st["iterations"], rank=orc.rank, active_fem_dofs=int(orc.active.size),
              full_relative_residual=float(np.linalg.norm(b - orc.H @ x) / bn) if bn else 0.0,
              woodbury_spd=M.spd)
    return x, st, orc, M
