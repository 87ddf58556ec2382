"""GPU assembly of the log-Neo-Hookean Tet4 Hessian into the solver's input form.

``FemAssembler`` wraps ``hsc_fem_assembler_*`` / ``hsc_fem_assemble``
(hsc_assemble.cu): the mesh analysis happens once, then every Newton step
assembles the FEM block of the system on the device from the current node
positions and per-tet Young's moduli, straight into a one-triangle BCOO the
solver reads (log_neo_hookean_3d.cu:62-135, global_linear_system.cu:215-248).

``CouplingAssembler`` wraps ``hsc_coupling_*`` (hsc_coupling.cu): the ABD-FEM
contact blocks J(xbar)^T H (abd_fem_linear_subsystem.cu:18-61) as sorted
upper-triangle BCOO blocks, together with the active FEM dofs and the dense
coupling E over them that the solver's setup extracts (linear_hsc.cu:205-247).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import HSCError

DT = 1.0 / 30.0


class FemAssembler:
    def __init__(self, tets, rest_x, rho=1000.0, nu=0.3, dt=DT, project=True):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        tets = np.ascontiguousarray(tets, dtype=np.int32)
        rest_x = np.ascontiguousarray(rest_x, dtype=np.float64)
        self.ntet, self.nnode = tets.shape[0], rest_x.shape[0]
        self._ptr = C.c_void_p()
        rc = self.lib.hsc_fem_assembler_create(tets.ctypes.data, self.ntet, self.nnode, rest_x.ctypes.data, rho, nu,
                                               dt, int(bool(project)), C.byref(self._ptr))
        if rc != _lib.HSC_OK:
            raise HSCError(rc, "hsc_fem_assembler_create failed")
        n = C.c_int64()
        self.lib.hsc_fem_pattern(self._ptr, None, None, C.byref(n))
        self.nnzb = n.value
        self.rows = torch.empty(self.nnzb, dtype=torch.int32, device="cuda")
        self.cols = torch.empty(self.nnzb, dtype=torch.int32, device="cuda")
        rc = self.lib.hsc_fem_pattern(self._ptr, C.c_void_p(self.rows.data_ptr()), C.c_void_p(self.cols.data_ptr()),
                                      C.byref(n))
        if rc != _lib.HSC_OK:
            raise HSCError(rc, "hsc_fem_pattern failed")

    def assemble(self, x, E, values=None, check=True):
        """Values (nnzb, 9) column-major blocks at positions x (nnode, 3) with moduli E (ntet,)."""
        torch = self.torch
        x = torch.as_tensor(x, dtype=torch.float64, device="cuda").contiguous()
        E = torch.as_tensor(E, dtype=torch.float64, device="cuda").contiguous()
        if E.numel() == 1:
            E = E.expand(self.ntet).contiguous()
        if values is None:
            values = torch.empty(self.nnzb, 9, dtype=torch.float64, device="cuda")
        inv = C.c_int32(0)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = self.lib.hsc_fem_assemble(self._ptr, C.c_void_p(x.data_ptr()), C.c_void_p(E.data_ptr()),
                                       C.c_void_p(values.data_ptr()), C.byref(inv) if check else None, stream)
        if rc != _lib.HSC_OK:
            raise HSCError(rc, f"hsc_fem_assemble failed ({inv.value} inverted tets)")
        return values

    def feasible_step(self, x0, dx, alpha0=1.0, max_halvings=60):
        """(alpha, halvings, limiting tets): the largest alpha0 * 2^-m whose segment keeps every
        tet's det F above 1e-8 (the reference's line-search feasibility rule)."""
        torch = self.torch
        x0 = torch.as_tensor(x0, dtype=torch.float64, device="cuda").contiguous()
        dx = torch.as_tensor(dx, dtype=torch.float64, device="cuda").contiguous()
        alpha, m, lim = C.c_double(), C.c_int32(), C.c_int32()
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = self.lib.hsc_fem_feasible_step(self._ptr, C.c_void_p(x0.data_ptr()), C.c_void_p(dx.data_ptr()),
                                            float(alpha0), int(max_halvings), C.byref(alpha), C.byref(m),
                                            C.byref(lim), stream)
        if rc not in (_lib.HSC_OK, _lib.HSC_ERR_NONSPD):
            raise HSCError(rc, "hsc_fem_feasible_step failed")
        return alpha.value, m.value, lim.value

    def close(self):
        if self._ptr:
            self.lib.hsc_fem_assembler_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CouplingAssembler:
    """ABD-FEM contact coupling on the device (see ``hsc_coupling_assemble``)."""

    def __init__(self, v2b, x_bar, nbody, nfem, body_fixed=None, fem_fixed=None, abd_block_offset=0,
                 fem_block_offset=None, p_first=True):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        v2b = np.ascontiguousarray(v2b, dtype=np.int32)
        x_bar = np.ascontiguousarray(x_bar, dtype=np.float64).reshape(-1, 3)
        self.nbody, self.nfem = int(nbody), int(nfem)
        self.qm = 12 * self.nbody
        self.fem_block_offset = 4 * self.nbody if fem_block_offset is None else int(fem_block_offset)
        bf = None if body_fixed is None else np.ascontiguousarray(body_fixed, dtype=np.int32)
        ff = None if fem_fixed is None else np.ascontiguousarray(fem_fixed, dtype=np.int32)
        self._ptr = C.c_void_p()
        rc = self.lib.hsc_coupling_assembler_create(
            len(v2b), v2b.ctypes.data, x_bar.ctypes.data, self.nbody, None if bf is None else bf.ctypes.data,
            self.nfem, None if ff is None else ff.ctypes.data, int(abd_block_offset), self.fem_block_offset,
            int(bool(p_first)), C.byref(self._ptr))
        if rc != _lib.HSC_OK:
            raise HSCError(rc, "hsc_coupling_assembler_create failed")

    def assemble(self, abd_vertex, fem_vertex, H):
        """dict(rows, cols, values (nblocks, 9) column-major, active (global dofs), E (qm, nactive))."""
        torch = self.torch
        av = torch.as_tensor(abd_vertex, dtype=torch.int32, device="cuda").contiguous()
        fv = torch.as_tensor(fem_vertex, dtype=torch.int32, device="cuda").contiguous()
        Hc = torch.as_tensor(H, dtype=torch.float64, device="cuda").reshape(-1, 9).contiguous()
        nb, na = C.c_int32(), C.c_int32()
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = self.lib.hsc_coupling_assemble(self._ptr, C.c_void_p(av.data_ptr()), C.c_void_p(fv.data_ptr()),
                                            C.c_void_p(Hc.data_ptr()), int(av.numel()), C.byref(nb), C.byref(na),
                                            stream)
        if rc != _lib.HSC_OK:
            raise HSCError(rc, "hsc_coupling_assemble failed")
        out = dict(rows=torch.empty(nb.value, dtype=torch.int32, device="cuda"),
                   cols=torch.empty(nb.value, dtype=torch.int32, device="cuda"),
                   values=torch.empty(nb.value, 9, dtype=torch.float64, device="cuda"),
                   active=torch.empty(na.value, dtype=torch.int32, device="cuda"),
                   E=torch.empty(self.qm, na.value, dtype=torch.float64, device="cuda"))
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t.numel() else None
        rc = self.lib.hsc_coupling_read(self._ptr, ptr(out["rows"]), ptr(out["cols"]), ptr(out["values"]),
                                        ptr(out["active"]), ptr(out["E"]), stream)
        if rc != _lib.HSC_OK:
            raise HSCError(rc, "hsc_coupling_read failed")
        return out

    def close(self):
        if self._ptr:
            self.lib.hsc_coupling_assembler_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
