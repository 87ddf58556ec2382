"""CPU oracle of the learned polynomial preconditioner.  TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import it.  It restates in NumPy (float64) what
``hsc_reimpl_b200/csrc/hsc_learned.cu`` computes on the GPU, so the tests
can check the CUDA kernels against it:

* ``bf16_round``      -- round-to-nearest-even FP32 -> BF16 (bit patterns);
* ``mlp_forward``     -- 16 -> 64 -> 64 -> 8, ReLU, softplus outputs;
* ``mlp_backward``    -- parameter gradients from dL/dw, summed over samples;
* ``poly_ls_loss``    -- L = sum_i tau_i (1 - theta_i q_w(theta_i))^2 and dL/dw;
* ``features``        -- the 16 per-system features from H, the DOF layout,
                         the coupling factors V, C and the previous-solve record;
* ``lanczos_measure`` -- Ritz values / Gauss weights of the CG Lanczos
                         tridiagonal (the spectral measure the loss uses);
* ``ls_teacher``      -- the non-negative least-squares weights of that loss.

The reference has no learned preconditioner (it fixes w_k = 1,
``reproduction/hsc_backend/linear_hsc.cu:330-343``); the MLP shape, loss and
features are this project's design, so parity here is GPU-vs-restatement.
"""
from __future__ import annotations

import numpy as np
from scipy.optimize import nnls

NF, NH, NO = 16, 64, 8
OFF_W1 = 0
OFF_B1 = OFF_W1 + NH * NF
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NO * NH
NPARAM = OFF_B3 + NO


def bf16_round(x):
    """FP32 values -> BF16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def bf16_to_float(b):
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(NH, NF), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(NH, NH),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(NO, NH), p[OFF_B3:NPARAM])


def softplus(o):
    return np.where(o > 20, o, np.log1p(np.exp(np.minimum(o, 20))))


def sigmoid(o):
    return 1.0 / (1.0 + np.exp(-o))


def mlp_forward(params, X):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    o = h2 @ W3.T + b3
    return h1, h2, o, softplus(o)


def mlp_backward(params, X, h1, h2, o, gw):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    go = gw * sigmoid(o)
    gz2 = (go @ W3) * (h2 > 0)
    gz1 = (gz2 @ W2) * (h1 > 0)
    g = np.zeros(NPARAM)
    g[OFF_W1:OFF_B1] = (gz1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = gz1.sum(0)
    g[OFF_W2:OFF_B2] = (gz2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = gz2.sum(0)
    g[OFF_W3:OFF_B3] = (go.T @ h2).ravel()
    g[OFF_B3:NPARAM] = go.sum(0)
    return g


def poly_basis(theta, degree=NO):
    """theta (..., m) -> theta (1 - theta)^k, shape (..., m, degree)."""
    th = np.asarray(theta, dtype=np.float64)[..., None]
    return th * (1.0 - th) ** np.arange(degree)


def poly_ls_loss(w, theta, tau, scale=1.0):
    Phi = poly_basis(theta, np.shape(w)[-1])             # (B, m, K)
    r = 1.0 - np.einsum("bmk,bk->bm", Phi, w)
    loss = scale * np.sum(tau * r * r, axis=1)
    gw = scale * (-2.0) * np.einsum("bm,bmk->bk", tau * r, Phi)
    return loss, gw


def lanczos_measure(alphas, betas, m):
    """Ritz values and Gauss weights (first eigenvector components squared) of
    the m x m Lanczos tridiagonal built from CG coefficients."""
    al = np.asarray(alphas, dtype=np.float64)[:m]
    be = np.asarray(betas, dtype=np.float64)[:m]
    m = al.size
    T = np.zeros((m, m))
    for j in range(m):
        T[j, j] = 1.0 / al[j] + (be[j - 1] / al[j - 1] if j > 0 else 0.0)
        if j + 1 < m:
            T[j, j + 1] = T[j + 1, j] = np.sqrt(be[j]) / al[j]
    th, U = np.linalg.eigh(T)
    return th, U[0] ** 2


def ls_teacher(theta, tau, degree=NO):
    """w >= 0 minimising sum_i tau_i (1 - theta_i q_w(theta_i))^2."""
    Phi = poly_basis(theta, degree)
    sw = np.sqrt(np.maximum(tau, 0.0))
    w, _ = nnls(Phi * sw[:, None], sw)
    return w


def _clamp(v):
    v = float(v)
    if not np.isfinite(v):
        return 0.0
    return min(8.0, max(-8.0, v))


def features(D, layout, active, V, C, prev=None):
    """The 16 features of hsc_learned.cu for the FEM block D (sparse, 3x3
    blocks), the active FEM dofs, the coupling factors V (a x k) and
    C = U^T P U (k x k), and the previous-solve record
    prev = (lambda_min, lambda_max, iterations, q0) or None."""
    import scipy.sparse as sp
    B = sp.csr_matrix(D).tobsr(blocksize=(3, 3))
    B.sort_indices()
    n = B.shape[0] // 3
    off = np.zeros(n)
    tr = np.zeros(n)
    for i in range(n):
        blocks = B.data[B.indptr[i]:B.indptr[i + 1]]
        cols = B.indices[B.indptr[i]:B.indptr[i + 1]]
        Dii = blocks[cols == i][0]
        tr[i] = np.trace(Dii)
        if np.linalg.det(Dii) > 0:
            inv = np.linalg.inv(Dii)
            off[i] = sum(np.linalg.norm(inv @ blk) for blk, c in zip(blocks, cols) if c != i)
    lt = np.where(tr > 0, np.log10(np.where(tr > 0, tr, 1.0)), 0.0)
    act_nodes = np.unique(np.asarray(active) // 3)
    a = len(active)
    k = V.shape[1] if V is not None and V.size else 0
    lr = float(np.trace(V @ C @ V.T)) if k else 0.0
    atr = float(tr[act_nodes].sum()) if act_nodes.size else 0.0
    rho = lr / atr if atr > 0 else 0.0
    f = np.zeros(NF)
    f[0] = np.log10(max(1, n)) / 5
    f[1] = 10.0 * a / max(1.0, 3.0 * n)
    f[2] = k / 128.0
    f[3] = off.mean()
    f[4] = np.sqrt(max(0.0, (off ** 2).mean() - off.mean() ** 2))
    f[5] = off.max() / 4
    f[6] = np.mean(off > 1.0)
    f[7] = (lt.max() - lt.min()) / 10
    f[8] = np.sqrt(max(0.0, (lt ** 2).mean() - lt.mean() ** 2)) / 3
    f[9] = off[act_nodes].mean() if act_nodes.size else 0.0
    f[10] = rho
    f[11] = np.log10(max(1.0 - rho, 1e-12)) / 6
    if prev is not None:
        lmin, lmax, iters, q0 = prev
        f[12] = 1.0
        f[13] = np.log10(max(lmin / max(q0, 1e-30), 1e-30)) / 6
        f[14] = np.log10(max(lmax, 1e-30))
        f[15] = np.log10(max(iters, 1.0)) / 4
    return np.array([_clamp(v) for v in f])
