"""CPU restatement of the ABD-FEM contact coupling assembly and of the HSC
solver's active-column / E extraction.  TEST INFRASTRUCTURE ONLY: the
checker for the device assembler, never called by the product.

* ``coupling_blocks`` follows ABDFEMLinearSubsystem_assemble_kernel
  (reproduction/hsc_backend/upstream/src/backends/cuda/coupling_system/
  abd_fem_linear_subsystem.cu:18-61): per contact (ABD vertex, FEM node,
  3x3 block H) the body rows get J(xbar)^T H, written as four 3x3 blocks
  (4 body + k, node); the block is zero when the body or the node is fixed.
  Duplicate (row, col) blocks are summed, as the global matrix's triplet
  conversion does (global_linear_system.cu:231-238), here in input order.
* ``extract`` follows linear_hsc.cu:216-247: the active FEM dofs are the
  three dofs of every node with a coupling block of nonzero squared norm,
  sorted; E is qm x a over them.

J(xbar) is libuipc's affine-body Jacobian (its ``ABDJacobi``, a header of the
un-vendored libuipc at the commit the reference pins): x = p + A xbar with
q = (p, rows of A); with ``p_first=False`` the order is (rows of A, p), that of
the reference's NumPy core (reproduction/core.py:201-206).
"""
from __future__ import annotations

import numpy as np


def jacobian(xbar, p_first=True):
    """3x12 map q -> x of an affine body at rest position xbar."""
    J = np.zeros((3, 12))
    for r in range(3):
        if p_first:
            J[r, r] = 1.0
            J[r, 3 + 3 * r:6 + 3 * r] = xbar
        else:
            J[r, 3 * r:3 * r + 3] = xbar
            J[r, 9 + r] = 1.0
    return J


def coupling_blocks(v2b, xbar, abd_vertex, fem_vertex, H, body_fixed=None, fem_fixed=None, p_first=True):
    """{(body, node): 12x3 sum of J^T H over the pair's contacts in input order}."""
    pairs = {}
    for t in range(len(abd_vertex)):
        v, f = int(abd_vertex[t]), int(fem_vertex[t])
        b = int(v2b[v])
        Ht = np.asarray(H[t], dtype=np.float64).reshape(3, 3, order="F") if np.ndim(H[t]) == 1 else H[t]
        blk = jacobian(xbar[v], p_first).T @ Ht
        fixed = (body_fixed is not None and body_fixed[b]) or (fem_fixed is not None and fem_fixed[f])
        if fixed:
            blk = np.zeros((12, 3))
        pairs[(b, f)] = pairs[(b, f)] + blk if (b, f) in pairs else blk
    return pairs


def bcoo(pairs, abd_block_offset, fem_block_offset):
    """Sorted upper-triangle BCOO (rows, cols, (n, 3, 3) blocks) of the pairs with a nonzero block."""
    ent = []
    for (b, f), blk in pairs.items():
        if not any(np.sum(blk[3 * k:3 * k + 3] ** 2) != 0 for k in range(4)):
            continue
        for k in range(4):
            ent.append((abd_block_offset + 4 * b + k, fem_block_offset + f, blk[3 * k:3 * k + 3]))
    ent.sort(key=lambda e: (e[0], e[1]))
    rows = np.array([e[0] for e in ent], dtype=np.int32)
    cols = np.array([e[1] for e in ent], dtype=np.int32)
    vals = np.array([e[2] for e in ent]).reshape(-1, 3, 3)
    return rows, cols, vals


def extract(pairs, nbody, fem_block_offset):
    """(active global dofs, E (12 nbody x a)) as linear_hsc.cu:216-247 builds them."""
    nodes = sorted({f for (b, f), blk in pairs.items()
                    if any(np.sum(blk[3 * k:3 * k + 3] ** 2) != 0 for k in range(4))})
    col = {f: i for i, f in enumerate(nodes)}
    E = np.zeros((12 * nbody, 3 * len(nodes)))
    for (b, f), blk in pairs.items():
        if f not in col:
            continue
        for k in range(4):
            B = blk[3 * k:3 * k + 3]
            if np.sum(B ** 2) == 0:
                continue
            E[12 * b + 3 * k:12 * b + 3 * k + 3, 3 * col[f]:3 * col[f] + 3] += B
    active = (3 * (fem_block_offset + np.array(nodes, dtype=np.int64))[:, None] + np.arange(3)).ravel()
    return active.astype(np.int32), E
