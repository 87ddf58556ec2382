"""Host-side mirror of the reference's linear-system plugin, over the C ABI.

``LinearHSC`` follows ``class LinearHSC : IterativeSolver``
(reproduction/hsc_backend/linear_hsc.cu:153-437):

* ``do_build(config)`` reads the same scene-config keys
  (linear_hsc.cu:172-193; defaults from the patch, integration.patch:33-54)
  and raises ``SimSystemException`` unless ``linear_system/solver`` is
  ``"linear_hsc"``;
* ``do_solve(info)`` takes a ``SolvingInfo``-like object with ``x()``,
  ``b()`` (device FP64 vectors) and ``A()`` (a device BCOO view) and the ABD /
  FEM dof ranges, runs one HSC solve on the GPU and raises ``HSCError`` on the
  conditions where the reference raises ``UIPC_ASSERT`` (no fallback);
* each solve appends the ``hsc_stats.jsonl`` record of linear_hsc.cu:420-431
  (plus this build's extra fields) when a workspace is set.

Device memory and streams come from PyTorch; every computation runs in
``libhsc_b200.so``.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from dataclasses import dataclass, field, fields

import numpy as np

from . import _lib
from ._lib import HSCError

PRECISIONS = {"fp64": _lib.HSC_FP64, "fp32": _lib.HSC_FP32, "bf16": _lib.HSC_BF16}
ABD_MODES = {"neumann": _lib.HSC_ABD_NEUMANN, "adaptive": _lib.HSC_ABD_ADAPTIVE, "exact": _lib.HSC_ABD_EXACT}


class SimSystemException(Exception):
    """The plugin is not selected (linear_hsc.cu:175-176)."""


@dataclass
class HSCOptions:
    max_rank: int = 128
    aca_rtol: float = 0.0
    neumann_order: int = 2
    omega: float = 0.7
    max_iter: int = 20000
    tol: float = 1e-6
    abd_inverse: str = "exact"
    abd_inverse_tol: float = 1e-5
    full_residual_limit: float = 0.1
    precision: str = "fp64"
    poly_weights: tuple | None = None      # set -> polynomial preconditioner with these weights
    poly_basis: str = "fem"                # "fem": terms on D (HSC_PRECOND_POLY); "schur": on S
    learned: bool = False                  # HSC_PRECOND_LEARNED (needs HSCContext.set_learned_model)
    block: bool = False                    # HSC_PRECOND_BLOCK (/ _BLOCK_LEARNED with learned=True)
    residual_replacement: int = 0
    refine_target: float = 0.0
    max_refinements: int = 20
    fallback_on_stall: bool = True
    threads_per_row: int = 0               # SpMV tile width 2, 4 or 8; 0: 4 resident, 2 streaming
    spin_limit: int = 20_000_000
    check_residual: bool = True
    trace_iterations: int = 0
    resident: bool = True                  # BSR slices + vector windows in shared memory when they fit
    fuse_update: bool = False              # resident mode: one grid barrier fewer per iteration
    aca_cluster: bool = True               # cluster ACA when the coupling fits; False: the grid kernel
    reorder: bool = True                   # internal FEM node renumbering into compact CTA parts
    aca_components: bool = True            # ACA per coupling component, merged (same factors as global)
    lanczos_stats: bool = False            # Ritz extremes of every solve (always on for the learned forms)
    coupled_part_weight: float = 1.2       # block forms: weight of the coupled parts' nodes in a second partition pass
    graph_replay: bool = False             # solve(): replay the captured CUDA graph (needs a non-default stream)

    @classmethod
    def reference(cls):
        """The reference plugin's defaults (linear_hsc.cu:162-164)."""
        return cls(neumann_order=5, max_iter=2000, abd_inverse="adaptive", tol=1e-4)

    def to_c(self) -> _lib.Options:
        o = _lib.Options()
        _lib.load().hsc_options_default(C.byref(o))
        o.max_rank = int(self.max_rank)
        o.aca_rtol = float(self.aca_rtol or 0.0)
        o.neumann_order = int(self.neumann_order)
        o.omega = float(self.omega)
        o.max_iter = int(self.max_iter)
        o.tol = float(self.tol)
        o.abd_inverse = ABD_MODES[self.abd_inverse]
        o.abd_inverse_tol = float(self.abd_inverse_tol)
        o.full_residual_limit = float(self.full_residual_limit)
        o.precision = PRECISIONS[self.precision]
        if self.block:
            # block-local polynomial with the exact coupling correction (pipelined PCG)
            if self.learned:
                o.preconditioner = _lib.HSC_PRECOND_BLOCK_LEARNED
            else:
                o.preconditioner = _lib.HSC_PRECOND_BLOCK
                w = [] if self.poly_weights is None else [float(v) for v in self.poly_weights]
                if len(w) > _lib.HSC_MAX_POLY:
                    raise ValueError("at most 16 polynomial weights")
                o.poly_degree = len(w)
                for i, v in enumerate(w):
                    o.poly_weights[i] = v
        elif self.learned:
            o.preconditioner = _lib.HSC_PRECOND_LEARNED
        elif self.poly_weights is not None:
            w = [float(v) for v in self.poly_weights]
            if not 1 <= len(w) <= _lib.HSC_MAX_POLY:
                raise ValueError("1..16 polynomial weights")
            if self.poly_basis not in ("fem", "schur"):
                raise ValueError("poly_basis is 'fem' or 'schur'")
            o.preconditioner = _lib.HSC_PRECOND_SCHUR_POLY if self.poly_basis == "schur" else _lib.HSC_PRECOND_POLY
            o.poly_degree = len(w)
            for i, v in enumerate(w):
                o.poly_weights[i] = v
        else:
            o.preconditioner = _lib.HSC_PRECOND_NEUMANN
        o.residual_replacement = int(self.residual_replacement)
        o.refine_target = float(self.refine_target or 0.0)
        o.max_refinements = int(self.max_refinements)
        o.fallback_on_stall = int(bool(self.fallback_on_stall))
        o.threads_per_row = int(self.threads_per_row)
        o.spin_limit = int(self.spin_limit)
        o.check_residual = int(bool(self.check_residual))
        o.trace_iterations = int(self.trace_iterations)
        o.resident = int(bool(self.resident))
        o.fuse_update = int(bool(self.fuse_update))
        o.aca_cluster = int(bool(self.aca_cluster))
        o.reorder = int(bool(self.reorder))
        o.aca_components = int(bool(self.aca_components))
        o.lanczos_stats = int(bool(self.lanczos_stats))
        o.coupled_part_weight = float(self.coupled_part_weight)
        o.graph_replay = int(bool(self.graph_replay))
        return o


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the HSC solver needs a CUDA device")
    return torch


@dataclass
class DeviceSystem:
    """One system resident on the GPU in the C-ABI input form."""
    rows: object
    cols: object
    values: object           # (nnzb, 9) column-major blocks, float64
    nblock: int
    layout: tuple
    b: object | None = None

    def bcoo(self) -> _lib.BCOO3:
        return _lib.BCOO3(self.rows.data_ptr(), self.cols.data_ptr(), self.values.data_ptr(),
                          int(self.rows.numel()), int(self.nblock))

    def c_layout(self) -> _lib.Layout:
        return _lib.Layout(*[int(v) for v in self.layout])

    @classmethod
    def from_system(cls, s, device="cuda"):
        torch = _torch()
        rows = torch.from_numpy(np.ascontiguousarray(s.rows, dtype=np.int32)).to(device)
        cols = torch.from_numpy(np.ascontiguousarray(s.cols, dtype=np.int32)).to(device)
        vals = torch.from_numpy(s.values_colmajor()).to(device)
        b = torch.from_numpy(np.ascontiguousarray(s.b, dtype=np.float64)).to(device)
        return cls(rows, cols, vals, s.nblock, tuple(s.layout), b)


class HSCContext:
    """Owns one hsc_ctx (grow-only device scratch, cached analysis)."""

    def __init__(self, options: HSCOptions | None = None):
        _torch()
        self.lib = _lib.load()
        self.options = options or HSCOptions()
        self._ptr = C.c_void_p()
        rc = self.lib.hsc_create(C.byref(self.options.to_c()), C.byref(self._ptr))
        if rc != _lib.HSC_OK:
            raise HSCError(rc, "hsc_create failed")

    def close(self):
        if self._ptr:
            self.lib.hsc_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, options: HSCOptions):
        rc = self.lib.hsc_set_options(self._ptr, C.byref(options.to_c()))
        self._check(rc)
        self.options = options

    def _check(self, rc):
        if rc != _lib.HSC_OK:
            raise HSCError(rc, self.lib.hsc_last_error(self._ptr).decode())

    def _stream(self, stream=None):
        torch = _torch()
        s = stream if stream is not None else torch.cuda.current_stream()
        return C.c_void_p(s.cuda_stream)

    def solve(self, ds: DeviceSystem, b=None, x=None, stream=None, raise_on_error=True):
        """x = HSC(A, b) on the GPU; returns (x, stats dict)."""
        torch = _torch()
        b = ds.b if b is None else b
        if x is None:
            x = torch.empty_like(b)
        st = _lib.Stats()
        rc = self.lib.hsc_solve(self._ptr, C.byref(ds.bcoo()), C.byref(ds.c_layout()), C.c_void_p(b.data_ptr()),
                                C.c_void_p(x.data_ptr()), self._stream(stream), C.byref(st))
        stats = st.as_dict()
        stats["status_name"] = _lib.STATUS_NAMES.get(rc, str(rc))
        if rc != _lib.HSC_OK and raise_on_error:
            self._check(rc)
        return x, stats

    def solve_batch(self, systems, xs=None, use_graph=False, stream=None, raise_on_error=True):
        torch = _torch()
        n = len(systems)
        A = (_lib.BCOO3 * n)(*[s.bcoo() for s in systems])
        L = (_lib.Layout * n)(*[s.c_layout() for s in systems])
        if xs is None:
            xs = [torch.empty_like(s.b) for s in systems]
        bp = (C.c_void_p * n)(*[s.b.data_ptr() for s in systems])
        xp = (C.c_void_p * n)(*[x.data_ptr() for x in xs])
        st = (_lib.Stats * n)()
        rc = self.lib.hsc_solve_batch(self._ptr, n, A, L, bp, xp, int(bool(use_graph)), self._stream(stream), st)
        stats = [s.as_dict() for s in st]
        if rc != _lib.HSC_OK and raise_on_error:
            self._check(rc)
        return xs, stats

    def spmv(self, ds: DeviceSystem, x, y=None, stream=None):
        """y = H x with the full symmetric H (IterativeSolver::spmv)."""
        torch = _torch()
        if y is None:
            y = torch.empty_like(x)
        rc = self.lib.hsc_spmv(self._ptr, C.byref(ds.bcoo()), C.byref(ds.c_layout()), C.c_void_p(x.data_ptr()),
                               C.c_void_p(y.data_ptr()), self._stream(stream))
        self._check(rc)
        return y

    def factors(self, sys_index=0):
        """(rank, U (qm x rank), V (a x rank), active dofs) of the last solve."""
        rank = C.c_int32()
        na = C.c_int32()
        self._check(self.lib.hsc_get_factors(self._ptr, sys_index, C.byref(rank), C.byref(na), None, 0, None, 0, None))
        k, a = rank.value, na.value
        qm = None
        act = np.zeros(max(a, 1), dtype=np.int32)
        self._check(self.lib.hsc_get_factors(self._ptr, sys_index, C.byref(rank), C.byref(na), None, 0, None, 0,
                                             act.ctypes.data))
        return k, a, act[:a]

    def partition(self, sys_index=0):
        """(perm, part_ptr) of the internal FEM node numbering: perm[i] = caller's node of internal
        node i; part p = internal nodes part_ptr[p] .. part_ptr[p + 1] - 1."""
        n, P = C.c_int32(), C.c_int32()
        self._check(self.lib.hsc_get_partition(self._ptr, sys_index, C.byref(n), C.byref(P), None, None))
        perm = np.zeros(max(n.value, 1), dtype=np.int32)
        ptr = np.zeros(P.value + 1, dtype=np.int32)
        self._check(self.lib.hsc_get_partition(self._ptr, sys_index, None, None, perm.ctypes.data, ptr.ctypes.data))
        return perm[:n.value], ptr

    def block_plan(self):
        """The block preconditioner's plan of the last block solve (hsc_debug_block_plan)."""
        keys = ("ctas", "R", "NS", "NCH", "W", "NA", "NCOL", "stage_vals", "NYC", "smem", "smem_y", "ncomp",
                "nslot", "kmax")
        out = np.zeros(len(keys), dtype=np.int64)
        self._check(self.lib.hsc_debug_block_plan(self._ptr, out.ctypes.data, len(keys)))
        return dict(zip(keys, (int(v) for v in out)))

    def factors_full(self, qm, sys_index=0):
        k, a, act = self.factors(sys_index)
        U = np.zeros((max(k, 1), qm))
        V = np.zeros((max(k, 1), max(a, 1)))
        self._check(self.lib.hsc_get_factors(self._ptr, sys_index, None, None, U.ctypes.data, qm, V.ctypes.data,
                                             max(a, 1), None))
        return U[:k].T.copy(), V[:k, :a].T.copy(), act

    def trace(self):
        """Per-CTA SM clocks at the PCG phase boundaries (options.trace_iterations > 0):
        array (ctas, iterations, 16)."""
        g, it = C.c_int32(), C.c_int32()
        self._check(self.lib.hsc_get_trace(self._ptr, None, 0, C.byref(g), C.byref(it)))
        out = np.zeros(g.value * it.value * 16, dtype=np.uint64)
        self._check(self.lib.hsc_get_trace(self._ptr, out.ctypes.data, out.size, None, None))
        return out.reshape(g.value, it.value, 16)

    def abd_inverse(self, qm, sys_index=0):
        P = np.zeros((qm, qm))
        self._check(self.lib.hsc_get_abd_inverse(self._ptr, sys_index, P.ctypes.data))
        return P

    # -- learned preconditioner -------------------------------------------------
    def set_learned_model(self, params_bf16):
        """Load the 5768 BF16 parameters (uint16 bit patterns) of the learned model."""
        p = np.ascontiguousarray(params_bf16, dtype=np.uint16)
        if p.size != _lib.HSC_MLP_PARAMS:
            raise ValueError(f"expected {_lib.HSC_MLP_PARAMS} parameters, got {p.size}")
        self._check(self.lib.hsc_set_learned_model(self._ptr, p.ctypes.data))

    def features(self, sys_index=0):
        """The 16 learned-model features of system `sys_index` after a solve."""
        out = np.zeros(_lib.HSC_FEATURES, dtype=np.float32)
        self._check(self.lib.hsc_get_features(self._ptr, sys_index, out.ctypes.data))
        return out

    def poly_weights(self, sys_index=0):
        """Polynomial weights the last solve used."""
        out = np.zeros(_lib.HSC_MAX_POLY)
        deg = C.c_int32()
        self._check(self.lib.hsc_get_poly_weights(self._ptr, sys_index, out.ctypes.data, out.size, C.byref(deg)))
        return out[:deg.value].copy()

    def lanczos(self, sys_index=0, max_pairs=256):
        """CG coefficients (alpha_k, beta_k) of the last solve, shape (pairs, 2)."""
        out = np.zeros((max_pairs, 2))
        n = C.c_int32()
        self._check(self.lib.hsc_get_lanczos(self._ptr, sys_index, out.ctypes.data, max_pairs, C.byref(n)))
        return out[:n.value].copy()


# ----------------------------------------------------------------------------
# the plugin mirror
# ----------------------------------------------------------------------------
# integration.patch:33-54.  "linear_system/solver" has no default here: the
# plugin is selected only by an explicit "linear_hsc" (linear_hsc.cu:174-176).
CONFIG_DEFAULTS = {
    "linear_system/tol_rate": 1e-4,
    "linear_system/hsc/max_rank": 128,
    "linear_system/hsc/neumann_order": 5,
    "linear_system/hsc/max_iter": 2000,
    "linear_system/hsc/adaptive_abd_inverse": 1,
    "linear_system/hsc/abd_inverse_tol": 1e-5,
    "linear_system/hsc/full_residual_limit": 0.1,
    "linear_system/hsc/omega": 0.7,
}


class SolvingInfo:
    """What GlobalLinearSystem::SolvingInfo hands a solver (global_linear_system.h:347-365):
    x() (written), b() (read), A() (one-triangle 3x3 BCOO), plus the ABD/FEM
    dof ranges the solver reads from its subsystems (linear_hsc.cu:197-198)."""

    def __init__(self, device_system: DeviceSystem, x=None):
        torch = _torch()
        self._ds = device_system
        self._x = x if x is not None else torch.zeros_like(device_system.b)
        self._iters = 0

    def x(self):
        return self._x

    def b(self):
        return self._ds.b

    def A(self):
        return self._ds

    def dof_layout(self):
        return self._ds.layout

    def iter_count(self, n=None):
        if n is not None:
            self._iters = int(n)
        return self._iters


class LinearHSC:
    """Drop-in for the reference's ``LinearHSC : IterativeSolver``."""

    def __init__(self, workspace: str | None = None, dump_systems: bool = False):
        self.workspace = workspace
        self.dump_systems = dump_systems      # <workspace>/systems/f<frame>_n<newton>.npz per solve
        self.ctx: HSCContext | None = None
        self.options: HSCOptions | None = None
        self.frame = 0
        self.newton = 0

    def do_build(self, config: dict, extra: HSCOptions | None = None):
        cfg = dict(CONFIG_DEFAULTS)
        cfg.update(config or {})
        if cfg.get("linear_system/solver") != "linear_hsc":
            raise SimSystemException("LinearHSC unused")
        o = extra or HSCOptions()
        o.max_rank = int(cfg["linear_system/hsc/max_rank"])
        o.neumann_order = int(cfg["linear_system/hsc/neumann_order"])
        o.max_iter = int(cfg["linear_system/hsc/max_iter"])
        o.omega = float(cfg["linear_system/hsc/omega"])
        adaptive = int(cfg["linear_system/hsc/adaptive_abd_inverse"])
        if extra is None or extra.abd_inverse != "exact":
            o.abd_inverse = "adaptive" if adaptive else "neumann"
        o.abd_inverse_tol = float(cfg["linear_system/hsc/abd_inverse_tol"])
        o.full_residual_limit = float(cfg["linear_system/hsc/full_residual_limit"])
        o.tol = float(cfg["linear_system/tol_rate"])
        if not (o.max_rank > 0 and o.neumann_order > 0 and o.max_iter > 0 and 0 < o.omega <= 1):
            raise ValueError("Invalid HSC parameters")            # linear_hsc.cu:188-189
        self.options = o
        self.ctx = HSCContext(o)

    def do_solve(self, info: SolvingInfo):
        x, stats = self.ctx.solve(info.A(), b=info.b(), x=info.x(), raise_on_error=False)
        info.iter_count(stats["pcg_iterations"])
        record = self.record(stats)
        if self.workspace:
            os.makedirs(self.workspace, exist_ok=True)
            with open(os.path.join(self.workspace, "hsc_stats.jsonl"), "a") as f:
                f.write(json.dumps(record) + "\n")
            if self.dump_systems:
                from .records import dump_system
                d = os.path.join(self.workspace, "systems")
                os.makedirs(d, exist_ok=True)
                dump_system(os.path.join(d, f"f{self.frame:06d}_n{self.newton:04d}.npz"), info.A(),
                            options=self.options, record=record, x=info.x())
        if stats["status"] != _lib.HSC_OK:
            raise HSCError(stats["status"], self.ctx.lib.hsc_last_error(self.ctx._ptr).decode())
        return stats

    def record(self, s):
        """The hsc_stats.jsonl record (linear_hsc.cu:420-431) plus extra fields."""
        prec = {v: k for k, v in PRECISIONS.items()}[s["precision"]]
        return {
            "frame": self.frame, "newton": self.newton, "fem_dofs": s["fem_dofs"], "abd_dofs": s["abd_dofs"],
            "active_fem_dofs": s["active_fem_dofs"], "rank": s["rank"],
            "aca_relative_error": s["aca_relative_error"], "pcg_iterations": s["pcg_iterations"],
            "schur_relative_residual": s["schur_relative_residual"],
            "full_relative_residual": s["full_relative_residual"], "setup_ms": s["setup_ms"],
            "total_ms": s["total_ms"], "active_mesh_contacts": 0, "active_ground_contacts": 0,
            "adaptive_abd_inverse": self.options.abd_inverse == "adaptive",
            "neumann_doublings": s["neumann_doublings"], "abd_inverse_residual": s["abd_inverse_residual"],
            "full_residual_limit": s["full_residual_limit"], "accepted": bool(s["accepted"]),
            "solver": "linear_hsc", "fallback": bool(s["fallback"]),
            "precision_mode": prec,
            "preconditioner": "polynomial" if s["preconditioner"] else "neumann",
            "refinement_steps": s["refinement_steps"], "pcg_ms": s["pcg_ms"],
            "lanczos_min": s["lanczos_min"], "lanczos_max": s["lanczos_max"],
        }


def solve_system(system, options: HSCOptions | None = None, ctx: HSCContext | None = None):
    """Upload a host ``HSCSystem`` and solve it; returns (x numpy, stats)."""
    ctx = ctx or HSCContext(options)
    if options is not None and ctx.options is not options:
        ctx.set_options(options)
    ds = DeviceSystem.from_system(system)
    x, stats = ctx.solve(ds, raise_on_error=False)
    return x.cpu().numpy(), stats, ctx
