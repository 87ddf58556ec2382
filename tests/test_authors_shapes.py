"""The build's kernels at the authors' kernel test shapes.

``reproduction/cuda_original.py`` (``validate``) compiles the authors' own kernels and
checks them in 20 seeded cases (numpy ``default_rng(2026)``) at 1e-10 absolute error
(``reproduction/results/gpu_checks.json``):

* ``spmv_sm_kernel<double, bs>`` (``sparse_matrix_square/spmv_cuda.cuh``) on a 2 x 2 block
  matrix of bs x bs blocks, bs = 3 and 12, against ``dense @ vec``;
* ``dmv_accumulate_kernel<double, bs>`` (``sparse_linear_solvers/conjugate_gradient_cuda.cuh``):
  ``z + 0.7 * blockdiag(diag) vec`` over 2 blocks.

The same random draws are made here in the same order.  The authors' SpMV takes a general
block matrix; this build's ``hsc_spmv`` takes one triangle of a symmetric H (libuipc's
input form), so the 2 x 2 block matrix is symmetrised (the diagonal blocks' symmetric parts
and the upper off-diagonal block mirrored) before it is stored as 3 x 3 blocks: bs = 3 is a
FEM-only system of 2 nodes, bs = 12 one affine body (12 dofs) coupled to 4 FEM nodes, so the
dense ABD block, the coupling block and the BSR block of ``hsc_spmv`` are all exercised.
``dmv_accumulate`` runs through ``hsc_debug_dmv_accumulate``, whose bs = 3 path is the PCG
kernel's block-Jacobi product.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _authors_draws(cases=20):
    """The inputs of cuda_original.validate's spmv / dmv checks, drawn in its order."""
    rng = np.random.default_rng(2026)
    out = []
    for _ in range(cases):
        rng.normal(size=(2, 3)); rng.normal(size=(2, 12)); rng.normal(size=3); rng.normal(size=(3, 3))
        per = {}
        for bs in (3, 12):
            blocks = rng.normal(size=(4, bs, bs))
            vec = rng.normal(size=2 * bs)
            diag, z = rng.normal(size=(2, bs, bs)), rng.normal(size=2 * bs)
            per[bs] = (blocks, vec, diag, z)
        out.append(per)
    return out


def _sym_dense(blocks):
    b0 = 0.5 * (blocks[0] + blocks[0].T)
    b3 = 0.5 * (blocks[3] + blocks[3].T)
    return np.block([[b0, blocks[1]], [blocks[1].T, b3]])


def _system(H, bs):
    from hsc_reimpl_b200.systems import HSCSystem, bcoo_upper_from_csr
    Hs = sp.csr_matrix(H)
    rows, cols, vals = bcoo_upper_from_csr(Hs)
    layout = (0, 0, 0, 6) if bs == 3 else (0, 12, 12, 12)
    n = H.shape[0]
    return HSCSystem("authors", layout, Hs, rows, cols, vals, np.zeros(n), np.zeros(n), {})


def test_spmv_at_the_authors_shapes():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200.solver import DeviceSystem, HSCContext
    ctx = HSCContext()
    worst = {3: 0.0, 12: 0.0}
    for per in _authors_draws():
        for bs, (blocks, vec, _, _) in per.items():
            H = _sym_dense(blocks)
            s = _system(H, bs)
            ds = DeviceSystem.from_system(s)
            y = ctx.spmv(ds, torch.from_numpy(vec).cuda()).cpu().numpy()
            worst[bs] = max(worst[bs], float(np.max(np.abs(y - H @ vec))))
    assert worst[3] < TOL and worst[12] < TOL, worst


def test_dmv_accumulate_at_the_authors_shapes():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200 import _lib
    lib = _lib.load()
    worst = {3: 0.0, 12: 0.0}
    for per in _authors_draws():
        for bs, (_, vec, diag, z) in per.items():
            planes = np.ascontiguousarray(diag.reshape(2, bs * bs).T)      # [(i*bs+j) * 2 + b]
            dp = torch.from_numpy(planes).cuda()
            dx = torch.from_numpy(vec).cuda()
            dz = torch.from_numpy(z.copy()).cuda()
            rc = lib.hsc_debug_dmv_accumulate(bs, 2, C.c_void_p(dp.data_ptr()), C.c_void_p(dx.data_ptr()),
                                              C.c_void_p(dz.data_ptr()), 0.7, None)
            torch.cuda.synchronize()
            assert rc == _lib.HSC_OK
            expected = z + 0.7 * np.einsum("bij,bj->bi", diag, vec.reshape(2, bs)).ravel()
            worst[bs] = max(worst[bs], float(np.max(np.abs(dz.cpu().numpy() - expected))))
    assert worst[3] < TOL and worst[12] < TOL, worst
