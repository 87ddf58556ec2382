"""CPU oracle of the FEM Hessian assembly.  TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import it.  It restates in NumPy the per-tet log-Neo-Hookean
Hessian of the reference and its assembly into a one-triangle BCOO:

* ``energy``, ``first_piola`` -- ``E`` and ``dEdF``, ``log_neo_hookean_function.h:77-91``;
* ``raw_hessian``  -- ``log_neo_hookean_function.h:93-104``: H[i+3a][j+3b] =
  mu d_ij d_ab + lambda G[i][a] G[j][b] - (lambda ln J - mu) G[i][b] G[j][a],
  G = cof(F)/J, column-major vec(F);
* ``spd``          -- ``ddEddF_spd`` (``log_neo_hookean_function.h:106-150``):
  the eigen-decomposition with negative eigenvalues clamped at 0 (here by
  LAPACK's symmetric solver instead of cyclic Jacobi);
* ``assemble``     -- ``log_neo_hookean_3d.cu:62-135``: F = Ds Dm^-1, the
  V dt^2 scaling, the shape-gradient pullback to the ten upper node blocks
  (the smaller node id first), summed over tets, plus the lumped mass
  rho V / 4; returned as sorted unique (row, col) blocks, column-major values
  (``global_linear_system.cu:215-248`` keeps one triangle).
"""
from __future__ import annotations

import numpy as np

MIN_JACOBIAN = 1e-8


def lame(E, nu):
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


def cofactor(F):
    C = np.empty_like(F)
    for i in range(3):
        for j in range(3):
            C[..., i, j] = (F[..., (i + 1) % 3, (j + 1) % 3] * F[..., (i + 2) % 3, (j + 2) % 3]
                            - F[..., (i + 1) % 3, (j + 2) % 3] * F[..., (i + 2) % 3, (j + 1) % 3])
    return C


def energy(F, mu, lam):
    """log-NH energy density psi = mu/2 (|F|^2 - 3) - mu ln J + lambda/2 (ln J)^2
    (``log_neo_hookean_function.h:77-83``); +inf unless det F > 1e-8."""
    J = np.linalg.det(F)
    with np.errstate(invalid="ignore", divide="ignore"):
        lnJ = np.log(J)
    psi = 0.5 * mu * (np.sum(F * F, axis=(-2, -1)) - 3.0) - mu * lnJ + 0.5 * lam * lnJ * lnJ
    return np.where(J > MIN_JACOBIAN, psi, np.inf)


def first_piola(F, mu, lam):
    """dpsi/dF = mu F + (lambda ln J - mu) cof(F) / J (``log_neo_hookean_function.h:85-91``)."""
    J = np.linalg.det(F)
    FinvT = np.swapaxes(np.linalg.inv(F), -1, -2)
    return mu[..., None, None] * F + (lam * np.log(J) - mu)[..., None, None] * FinvT


def raw_hessian(F, mu, lam):
    J = np.linalg.det(F)
    G = cofactor(F) / J[:, None, None]
    q = lam * np.log(J) - mu
    H = np.zeros((F.shape[0], 3, 3, 3, 3))  # [t, a, i, b, j] for H[i + 3a][j + 3b]
    eye = np.eye(3)
    H += mu[:, None, None, None, None] * np.einsum("ij,ab->aibj", eye, eye)[None]
    H += lam[:, None, None, None, None] * np.einsum("tia,tjb->taibj", G, G)
    H -= q[:, None, None, None, None] * np.einsum("tib,tja->taibj", G, G)
    return H.reshape(-1, 9, 9)


def spd(H):
    w, Q = np.linalg.eigh(H)
    return np.einsum("tik,tk,tjk->tij", Q, np.maximum(w, 0.0), Q)


def assemble(tets, rest_x, x, E, rho=1000.0, nu=0.3, dt=1.0 / 30.0, project=True):
    """(rows, cols, values (nnzb, 9) column-major) of the FEM Hessian's upper block triangle."""
    tets = np.asarray(tets, dtype=np.int64)
    n = rest_x.shape[0]
    Dm = np.transpose(rest_x[tets[:, 1:]] - rest_x[tets[:, :1]], (0, 2, 1))
    vol = np.abs(np.linalg.det(Dm)) / 6.0
    Dminv = np.linalg.inv(Dm)
    Ds = np.transpose(x[tets[:, 1:]] - x[tets[:, :1]], (0, 2, 1))
    F = Ds @ Dminv
    E = np.broadcast_to(np.asarray(E, dtype=np.float64), (tets.shape[0],))
    mu, lam = lame(E, nu)
    H = raw_hessian(F, mu, lam)
    if project:
        H = spd(H)
    H = H.reshape(-1, 3, 3, 3, 3)
    Gs = np.concatenate([-Dminv.sum(1, keepdims=True), Dminv], 1)      # (t, node, a)
    K = np.einsum("tka,tlb,taibj->tkilj", Gs, Gs, H) * (vol * dt * dt)[:, None, None, None, None]
    blocks = {}
    for u in range(4):
        for v in range(u, 4):
            L = np.where(tets[:, u] <= tets[:, v], u, v)
            R = np.where(tets[:, u] <= tets[:, v], v, u)
            B = K[np.arange(len(tets)), L, :, R, :]                       # (t, i, j)
            keys = tets[np.arange(len(tets)), L] * n + tets[np.arange(len(tets)), R]
            for kk, b in zip(keys, B):
                blocks[kk] = blocks.get(kk, 0.0) + b
    mass = np.zeros(n)
    np.add.at(mass, tets.ravel(), np.repeat(rho * vol / 4.0, 4))
    for i in range(n):
        blocks[i * n + i] = blocks.get(i * n + i, 0.0) + mass[i] * np.eye(3)
    keys = np.array(sorted(blocks))
    vals = np.array([np.asarray(blocks[k]).T.reshape(9) for k in keys])  # column-major
    return (keys // n).astype(np.int32), (keys % n).astype(np.int32), vals


def _triple(a, b, c):
    return a @ np.cross(b, c)


def segment_feasible(A, E):
    """``feasible_segment`` (``log_neo_hookean_function.h:37-75``): det(A + s (E - A))
    stays above 1e-8 on [0, 1] -- endpoints and the derivative roots of the cubic."""
    B = E - A
    c0 = np.linalg.det(A)
    c1 = _triple(B[:, 0], A[:, 1], A[:, 2]) + _triple(A[:, 0], B[:, 1], A[:, 2]) + _triple(A[:, 0], A[:, 1], B[:, 2])
    c2 = _triple(A[:, 0], B[:, 1], B[:, 2]) + _triple(B[:, 0], A[:, 1], B[:, 2]) + _triple(B[:, 0], B[:, 1], A[:, 2])
    c3 = np.linalg.det(B)
    if not (c0 > MIN_JACOBIAN and np.linalg.det(E) > MIN_JACOBIAN):
        return False
    a, b, c = 3 * c3, 2 * c2, c1
    roots = []
    scale = abs(a) + abs(b) + abs(c)
    eps = 32 * 2.220446049250313e-16 * scale
    if abs(a) <= eps:
        if abs(b) > eps:
            roots.append(-c / b)
    else:
        disc = b * b - 4 * a * c
        if disc >= 0:
            q = -0.5 * (b + np.copysign(np.sqrt(disc), b))
            roots += [-b / (2 * a)] if q == 0 else [q / a, c / q]
    return all(not (0 < s < 1) or ((c3 * s + c2) * s + c1) * s + c0 > MIN_JACOBIAN for s in roots)


def feasible_step(tets, rest_x, x0, dx, alpha0=1.0, max_halvings=60):
    """(alpha, halvings, limiting tets) of the backtracking rule: the fewest halvings of alpha0
    that keep every tet's segment feasible."""
    tets = np.asarray(tets)
    Dminv = np.linalg.inv(np.transpose(rest_x[tets[:, 1:]] - rest_x[tets[:, :1]], (0, 2, 1)))
    worst, limited = 0, 0
    for t, nd in enumerate(tets):
        F0 = np.transpose(x0[nd[1:]] - x0[nd[:1]]) @ Dminv[t]
        s, m = alpha0, 0
        while m <= max_halvings:
            xs = x0[nd] + s * dx[nd]
            F1 = np.transpose(xs[1:] - xs[:1]) @ Dminv[t]
            if segment_feasible(F0, F1):
                break
            m += 1
            s *= 0.5
        worst = max(worst, m)
        limited += m > 0
    if worst > max_halvings:
        return 0.0, worst, limited
    return alpha0 * 2.0 ** -worst, worst, limited
