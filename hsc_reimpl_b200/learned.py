"""Learned polynomial preconditioner: the training systems, training on the
GPU with the library's own kernels, evaluation, and the model file.

The preconditioner (``HSC_PRECOND_LEARNED``, hsc_learned.cu) replaces the
reference's fixed Neumann weights (w_k = 1, linear_hsc.cu:330-343) by 8
positive weights of a Schur-basis polynomial, z = sum_k w_k t_k with
t_k = (I - w Dd^-1 S)^k w Dd^-1 r, chosen per system by a 16-64-64-8 MLP from
features computed on the device (hsc_get_features).

Training data come from the solver itself, along seeded "trajectories" of the
vehicle-scale system: the build has no Newton integrator, so a trajectory is a
seeded sequence of vehicle systems whose ground-tire Young's moduli random-walk
in [1e6, 1e8] Pa and whose tread contact patches roll, change size (5-15 % of
the tread) and change barrier stiffness from step to step.  For every system:

1. a 16-step Lanczos probe (PCG with the plain Jacobi preconditioner) gives the
   Ritz values theta_i and Gauss weights tau_i of w Dd^-1 S seen from the
   right-hand side -- enough to integrate the degree-18 loss exactly;
2. the least-squares teacher weights (non-negative, fitted to that measure)
   precondition a full solve, whose Lanczos record becomes the next step's
   "previous solve" features, as in deployment;
3. the features of the system are read back.

The MLP is trained to minimise L(w) = sum_i tau_i (1 - theta_i q_w(theta_i))^2
directly (hsc_mlp_forward / hsc_poly_ls_loss / hsc_mlp_backward /
hsc_adam_step); BF16 parameters with FP32 master copies and accumulation.
"""
from __future__ import annotations

import ctypes as C
import json
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib
from . import systems as S

HERE = Path(__file__).resolve().parent
MODEL_PATH = HERE / "learned_poly_model.npz"
NF, NH, NO = _lib.HSC_FEATURES, _lib.HSC_MLP_HIDDEN, _lib.HSC_MLP_OUT
NPARAM = _lib.HSC_MLP_PARAMS
OFF_B3 = NPARAM - NO
OFF_W3 = OFF_B3 - NO * NH
PROBE_STEPS = 16


# ----------------------------------------------------------------------------
# vehicle trajectories
# ----------------------------------------------------------------------------
def _block_triplets(r, c, v):
    """Scalar triplets of a symmetric part -> (block key row, block col, element, value) of its
    upper block triangle, element e = (r % 3) + 3 (c % 3) (column-major 3x3)."""
    br, bc = r // 3, c // 3
    keep = br <= bc
    return br[keep], bc[keep], (r[keep] % 3) + 3 * (c[keep] % 3), v[keep]


class VehicleBase:
    """Fixed part of the vehicle system at one set of node positions: FEM mass,
    per-tire elastic Hessians at E = 1 (the log-NH Hessian and its SPD
    projection are linear in E), rims, spindles and joints, all reduced to
    value vectors over one upper block pattern."""

    def __init__(self, variant=0, nr=4, na=5, nc=93, nu=0.3, rho=1000.0, E_abd=1e10, k_rim=1e7, k_joint=1e9,
                 perturb=0.02):
        rng = np.random.default_rng(10_000 + variant)
        self.ntire, nbody = 7, 12
        meshes = []
        for t in range(self.ntire):
            center = np.array([1.2 * (t % 4), 0.5 * (t // 4), 0.0])
            x, tets, _ = S.annulus_mesh(nr=nr, na=na, nc=nc, center=center)
            meshes.append((x, tets, center))
        self.nodes_per = meshes[0][0].shape[0]
        nn = self.ntire * self.nodes_per
        self.qm, self.fn = 12 * nbody, 3 * nn
        self.nblock = (self.qm + self.fn) // 3
        qm = self.qm
        parts = {"mass": [], "fixed": []}
        for t in range(self.ntire):
            parts[f"el{t}"] = []
        self.x = np.zeros((nn, 3))
        self.centers = []
        self.tread = []
        for t, (x, tets, center) in enumerate(meshes):
            base = t * self.nodes_per
            self.x[base:base + self.nodes_per] = x
            self.centers.append(center)
            r, c, v, _ = S.fem_hessian(x, tets, 1.0, nu, rho, perturb=perturb, rng=rng)
            nm = 3 * self.nodes_per                      # the lumped mass diagonal is appended last
            parts[f"el{t}"].append((qm + 3 * base + r[:-nm], qm + 3 * base + c[:-nm], v[:-nm]))
            parts["mass"].append((qm + 3 * base + r[-nm:], qm + 3 * base + c[-nm:], v[-nm:]))
            rim = [((0 * (na + 1) + ia) * nc + ic) for ia in (0, na) for ic in range(0, nc, 5)]
            asm = S._Assembler(qm + self.fn)
            asm.add_dense(12 * t + np.arange(12), S.abd_block(20.0, x[rim] - center, E_abd,
                                                              np.pi * 0.27 ** 2 * 0.3 * 0.1))
            for node in rim:
                S._stitch(asm, qm, base + node, t, x[node] - center, k_rim)
            parts["fixed"].append((np.concatenate(asm.r), np.concatenate(asm.c), np.concatenate(asm.v)))
            self.tread.append(base + np.array([((nr * (na + 1) + ia) * nc + ic) for ia in range(na + 1)
                                               for ic in range(nc)]))
        asm = S._Assembler(qm + self.fn)
        for s in range(4):
            pts = rng.uniform(-0.1, 0.1, (16, 3))
            asm.add_dense(12 * (7 + s) + np.arange(12), S.abd_block(10.0, pts, E_abd, 0.004))
            for p in (np.array([0.0, 0.1, 0.0]), np.array([0.05, 0.1, 0.05]), np.array([0.0, 0.1, 0.08])):
                S._joint(asm, 7 + s, p, s, p + np.array([0.0, -0.25, 0.0]), k_joint)
        for s in range(3):
            S._joint(asm, 7 + s, np.array([0.3, 0.0, 0.0]), 8 + s, np.array([-0.3, 0.0, 0.0]), 1e-2 * k_joint)
        gpts = rng.uniform(-2.0, 2.0, (32, 3))
        asm.add_dense(12 * 11 + np.arange(12), S.abd_block(1e4, gpts, E_abd, 10.0))
        parts["fixed"].append((np.concatenate(asm.r), np.concatenate(asm.c), np.concatenate(asm.v)))
        # one upper block pattern for everything fixed
        trip = {}
        keys = []
        for name, lst in parts.items():
            r = np.concatenate([p[0] for p in lst]).astype(np.int64)
            c = np.concatenate([p[1] for p in lst]).astype(np.int64)
            v = np.concatenate([p[2] for p in lst])
            br, bc, e, vv = _block_triplets(r, c, v)
            trip[name] = (br * self.nblock + bc, e, vv)
            keys.append(trip[name][0])
        self.keys = np.unique(np.concatenate(keys))
        nb = self.keys.size
        self.vec = {}
        for name, (k, e, v) in trip.items():
            pos = np.searchsorted(self.keys, k) * 9 + e
            self.vec[name] = np.bincount(pos, weights=v, minlength=9 * nb).reshape(nb, 9)
        self.ground_body = 11
        self.ground_point = np.array([1.8, 0.25, -1.0])


class VehicleTrajectory:
    """A seeded sequence of vehicle systems over one VehicleBase (see the module docstring)."""

    E_CARRIED = 1e10

    def __init__(self, base: VehicleBase, seed: int, steps: int = 300, contact_every: int = 10,
                 k_range=(1e6, 1e9)):
        self.base, self.seed, self.steps, self.every = base, seed, steps, contact_every
        self.k_range = k_range

    def __iter__(self):
        """Yields (step, rows int32, cols int32, values (nnzb, 9) float64, meta dict)."""
        B = self.base
        rng = np.random.default_rng(seed=[7, self.seed])
        logE = rng.uniform(6.0, 8.0, 3)
        speed = rng.uniform(0.002, 0.01, B.ntire)
        th0 = rng.uniform(0, 2 * np.pi, B.ntire)
        frac = rng.uniform(0.05, 0.15, B.ntire)
        fem_b0 = B.qm // 3
        for step in range(self.steps):
            if step % self.every == 0:
                frac = np.clip(frac + rng.normal(0, 0.01, B.ntire), 0.05, 0.15)
                nodes, nrm, logk = [], [], []
                for t in range(B.ntire):
                    tread = B.tread[t]
                    c = B.centers[t]
                    count = max(1, int(round(frac[t] * tread.size)))
                    ang = np.arctan2(B.x[tread, 2] - c[2], B.x[tread, 0] - c[0])
                    dist = np.abs(np.angle(np.exp(1j * (ang - th0[t]))))
                    patch = tread[np.argsort(dist, kind="stable")[:count]]
                    nv = B.x[patch] - c
                    nv[:, 1] = 0.0
                    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
                    nv += 0.05 * rng.standard_normal(nv.shape)
                    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
                    nodes.append(patch)
                    nrm.append(nv)
                    logk.append(rng.uniform(np.log(self.k_range[0]), np.log(self.k_range[1]), patch.size))
                nodes = np.concatenate(nodes)
                nrm = np.concatenate(nrm)
                logk = np.concatenate(logk)
                order = np.argsort(nodes)
                nodes, nrm, logk = nodes[order], nrm[order], logk[order]
                # window pattern: the fixed blocks plus the ground body's coupling blocks
                gb = 4 * B.ground_body
                ck = ((gb + np.arange(4))[:, None] * B.nblock + (fem_b0 + nodes)[None, :]).ravel()
                allk = np.concatenate([B.keys, ck])
                perm = np.argsort(allk, kind="stable")
                inv = np.empty_like(perm)
                inv[perm] = np.arange(perm.size)
                keys = allk[perm]
                base_pos = inv[:B.keys.size]
                cpl_pos = inv[B.keys.size:].reshape(4, -1)
                rows = (keys // B.nblock).astype(np.int32)
                cols = (keys % B.nblock).astype(np.int32)
                diag_pos = np.searchsorted(keys, (fem_b0 + nodes) * B.nblock + fem_b0 + nodes)
                gdiag = np.array([[np.searchsorted(keys, (gb + a) * B.nblock + gb + b) if a <= b else -1
                                   for b in range(4)] for a in range(4)])
            logE = np.clip(logE + rng.normal(0, 0.05, 3), 6.0, 8.0)
            logk = np.clip(logk + rng.normal(0, 0.2, logk.size), np.log(self.k_range[0]), np.log(self.k_range[1]))
            k = np.exp(logk)
            E = np.concatenate([np.full(4, self.E_CARRIED), 10.0 ** logE])
            vb = B.vec["mass"] + B.vec["fixed"]
            for t in range(B.ntire):
                vb = vb + E[t] * B.vec[f"el{t}"]
            vals = np.zeros((keys.size, 9))
            vals[base_pos] = vb
            # contacts: H += k g g^T, g = [n at the node, -P^T n on the ground body]
            Pn = np.zeros((nodes.size, 12))
            rest = B.x[nodes] - B.ground_point
            for r in range(3):
                Pn[:, 3 * r:3 * r + 3] = nrm[:, r:r + 1] * rest
                Pn[:, 9 + r] = nrm[:, r]
            gq = -Pn                                              # (c, 12)
            nnT = k[:, None, None] * nrm[:, :, None] * nrm[:, None, :]
            np.add.at(vals, diag_pos, np.transpose(nnT, (0, 2, 1)).reshape(-1, 9))
            for q in range(4):                                    # coupling blocks, ABD rows 3q..3q+2
                blk = k[:, None, None] * gq[:, 3 * q:3 * q + 3, None] * nrm[:, None, :]
                vals[cpl_pos[q]] += np.transpose(blk, (0, 2, 1)).reshape(-1, 9)
            Q = np.einsum("c,ci,cj->ij", k, gq, gq)               # ground-body 12x12
            for a in range(4):
                for b in range(a, 4):
                    vals[gdiag[a, b]] += Q[3 * a:3 * a + 3, 3 * b:3 * b + 3].T.reshape(9)
            th0 = th0 + speed
            yield step, rows, cols, vals, dict(E=E, contact_nodes=nodes, normals=nrm, k=k, nnzb=int(keys.size))

    def layout(self):
        return (0, self.base.qm, self.base.qm, self.base.fn)


# ----------------------------------------------------------------------------
# model parameters
# ----------------------------------------------------------------------------
def bf16_bits(x):
    """FP32 -> BF16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_values(b):
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def init_params(seed=0):
    """He-initialised hidden layers; the output layer starts at w_k = 1 (the
    Schur-basis Neumann series) with small weights."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    p[0:NH * NF] = rng.normal(0, np.sqrt(2.0 / NF), NH * NF)
    o = NH * NF + NH
    p[o:o + NH * NH] = rng.normal(0, np.sqrt(2.0 / NH), NH * NH)
    p[OFF_W3:OFF_B3] = rng.normal(0, 0.01, NO * NH)
    p[OFF_B3:] = np.log(np.expm1(1.0))
    return p


def save_model(path, params_fp32, meta):
    np.savez(path, params_bf16=bf16_bits(params_fp32), meta=json.dumps(meta))


def load_model(path=MODEL_PATH):
    """(BF16 bit patterns, metadata dict) of a saved model."""
    z = np.load(path)
    return z["params_bf16"], json.loads(str(z["meta"]))


# ----------------------------------------------------------------------------
# dataset generation (GPU)
# ----------------------------------------------------------------------------
@dataclass
class Sample:
    features: np.ndarray
    theta: np.ndarray
    tau: np.ndarray
    teacher: np.ndarray
    teacher_iters: int


def lanczos_measure(coef):
    """Ritz values and Gauss weights of the CG Lanczos tridiagonal from (alpha, beta) pairs."""
    al, be = coef[:, 0], coef[:, 1]
    m = al.size
    T = np.zeros((m, m))
    for j in range(m):
        T[j, j] = 1.0 / al[j] + (be[j - 1] / al[j - 1] if j > 0 else 0.0)
        if j + 1 < m:
            T[j, j + 1] = T[j + 1, j] = np.sqrt(max(be[j], 0.0)) / al[j]
    th, U = np.linalg.eigh(T)
    return th, U[0] ** 2


def ls_weights(theta, tau, degree=NO):
    """Non-negative least-squares weights of sum_i tau_i (1 - theta_i q_w(theta_i))^2."""
    from scipy.optimize import nnls
    Phi = theta[:, None] * (1.0 - theta[:, None]) ** np.arange(degree)
    sw = np.sqrt(np.maximum(tau, 0.0))
    w, _ = nnls(Phi * sw[:, None], sw)
    if not np.any(w > 0):
        w = np.ones(degree)
    return w


class SystemFeeder:
    """Uploads trajectory steps as DeviceSystems (values, rhs = H x* / |H x*|)."""

    def __init__(self, ctx, layout, device="cuda"):
        import torch
        self.torch = torch
        self.ctx, self.layout, self.device = ctx, layout, device
        self.rows = self.cols = None
        self._key = None

    def device_system(self, rows, cols, vals, nblock, seed):
        from .solver import DeviceSystem
        torch = self.torch
        if self._key is not rows:
            self.rows = torch.from_numpy(rows).to(self.device)
            self.cols = torch.from_numpy(cols).to(self.device)
            self._key = rows
        v = torch.from_numpy(np.ascontiguousarray(vals)).to(self.device)
        g = torch.Generator(device="cpu").manual_seed(int(seed))
        xs = torch.randn(3 * nblock, generator=g, dtype=torch.float64).to(self.device)
        ds = DeviceSystem(self.rows, self.cols, v, nblock, self.layout, None)
        b = self.ctx.spmv(ds, xs)
        ds.b = b / torch.linalg.vector_norm(b)
        return ds


def generate(trajectories, probe_steps=PROBE_STEPS, log=None):
    """Run the solver along the trajectories; returns a dict of arrays
    (features, theta, tau, teacher weights, teacher iterations, meta)."""
    from .solver import HSCContext, HSCOptions
    probe_opt = HSCOptions(neumann_order=1, max_iter=probe_steps, tol=0.0, check_residual=False)
    ctx_probe = HSCContext(probe_opt)
    feats, thetas, taus, teach, iters = [], [], [], [], []
    t0 = time.time()
    for ti, traj in enumerate(trajectories):
        ctx_main = HSCContext(HSCOptions())          # a fresh previous-solve record per trajectory
        lay = traj.layout()
        feeder = SystemFeeder(ctx_probe, lay)
        for step, rows, cols, vals, meta in traj:
            ds = feeder.device_system(rows, cols, vals, traj.base.nblock, seed=traj.seed * 1000 + step)
            ctx_probe.solve(ds, raise_on_error=False)
            coef = ctx_probe.lanczos()
            th, tau = lanczos_measure(coef)
            w = ls_weights(th, tau)
            ctx_main.set_options(HSCOptions(poly_weights=tuple(w), poly_basis="schur", fallback_on_stall=True))
            _, st = ctx_main.solve(ds, raise_on_error=False)
            feats.append(ctx_main.features())
            m = th.size
            thp = np.zeros(probe_steps); tap = np.zeros(probe_steps)
            thp[:m], tap[:m] = th, tau / max(tau.sum(), 1e-300)
            thetas.append(thp); taus.append(tap); teach.append(w); iters.append(st["pcg_iterations"])
        if log:
            log(f"trajectory {ti} ({traj.seed}): {len(feats)} systems, {time.time() - t0:.0f} s, "
                f"teacher iterations median {int(np.median(iters[-traj.steps:]))}")
    return dict(features=np.array(feats, np.float32), theta=np.array(thetas, np.float32),
                tau=np.array(taus, np.float32), teacher=np.array(teach), teacher_iters=np.array(iters))


# ----------------------------------------------------------------------------
# training (GPU, the library's kernels)
# ----------------------------------------------------------------------------
class Trainer:
    """Adam on FP32 master parameters, BF16 working copy, mean LS-polynomial loss."""

    def __init__(self, params_fp32, device="cuda", lr=1e-3, seed=0):
        import torch
        self.torch, self.dev, self.lr = torch, device, lr
        self.lib = _lib.load()
        self.master = torch.from_numpy(np.asarray(params_fp32, np.float32).copy()).to(device)
        self.pbf = torch.from_numpy(bf16_bits(params_fp32).view(np.int16)).to(device)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.grad = torch.zeros_like(self.master)
        self.step_no = 0
        self.gen = torch.Generator(device="cpu").manual_seed(seed)
        self._cap = 0

    def _buffers(self, B):
        torch = self.torch
        if B > self._cap:
            f = dict(dtype=torch.float32, device=self.dev)
            self.h1 = torch.empty(B, NH, **f)
            self.h2 = torch.empty(B, NH, **f)
            self.o = torch.empty(B, NO, **f)
            self.w = torch.empty(B, NO, **f)
            self.gw = torch.empty(B, NO, **f)
            self.loss = torch.empty(B, **f)
            self.scratch = torch.empty(B * (NO + 2 * NH), **f)
            self._cap = B

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr())

    def forward(self, X, B):
        self._buffers(B)
        s = C.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        rc = self.lib.hsc_mlp_forward(self._p(self.pbf), self._p(X), B, self._p(self.h1), self._p(self.h2),
                                      self._p(self.o), self._p(self.w), s)
        assert rc == 0, rc
        return self.w[:B]

    def loss_and_grad(self, X, TH, TAU):
        """Mean loss over the batch and the parameter gradient (in self.grad)."""
        B, m = TH.shape
        self.forward(X, B)
        s = C.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        rc = self.lib.hsc_poly_ls_loss(self._p(self.w), self._p(TH), self._p(TAU), B, m, C.c_float(1.0 / B),
                                       self._p(self.loss), self._p(self.gw), s)
        assert rc == 0, rc
        rc = self.lib.hsc_mlp_backward(self._p(self.pbf), self._p(X), self._p(self.h1), self._p(self.h2),
                                       self._p(self.o), self._p(self.gw), B, self._p(self.scratch),
                                       self._p(self.grad), s)
        assert rc == 0, rc
        return self.loss[:B]

    def step(self, X, TH, TAU):
        loss = self.loss_and_grad(X, TH, TAU)
        self.step_no += 1
        s = C.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        rc = self.lib.hsc_adam_step(self._p(self.master), self._p(self.pbf), self._p(self.grad), self._p(self.m),
                                    self._p(self.v), NPARAM, C.c_float(self.lr), C.c_float(0.9),
                                    C.c_float(0.999), C.c_float(1e-8), C.c_float(0.0), self.step_no, s)
        assert rc == 0, rc
        return loss

    def fit(self, data, epochs=200, batch=512, val=None, log=None):
        torch = self.torch
        X = torch.from_numpy(data["features"]).to(self.dev)
        TH = torch.from_numpy(data["theta"]).to(self.dev)
        TAU = torch.from_numpy(data["tau"]).to(self.dev)
        n = X.shape[0]
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=self.gen).to(self.dev)
            tot = 0.0
            for i in range(0, n, batch):
                idx = perm[i:i + batch]
                loss = self.step(X[idx].contiguous(), TH[idx].contiguous(), TAU[idx].contiguous())
                tot += float(loss.sum())
            rec = {"epoch": ep, "train_loss": tot / max(1, (n + batch - 1) // batch)}
            if val is not None and (ep % 10 == 9 or ep == epochs - 1):
                rec["val_loss"] = self.evaluate_loss(val)
            hist.append(rec)
            if log and (ep % 10 == 9 or ep == epochs - 1):
                log(json.dumps(rec))
        return hist

    def evaluate_loss(self, data):
        torch = self.torch
        X = torch.from_numpy(data["features"]).to(self.dev)
        TH = torch.from_numpy(data["theta"]).to(self.dev)
        TAU = torch.from_numpy(data["tau"]).to(self.dev)
        loss = self.loss_and_grad(X, TH, TAU)
        return float(loss.sum())

    def params_fp32(self):
        return self.master.cpu().numpy()


# ----------------------------------------------------------------------------
# evaluation
# ----------------------------------------------------------------------------
def evaluate(params_bf16, trajectories, log=None, precision="fp64"):
    """Per system: PCG iterations and PCG time to 1e-6 with the learned
    preconditioner, plain order-2 Neumann (the reference form) and the
    Schur-basis Neumann series of the same degree."""
    from .solver import HSCContext, HSCOptions
    modes = {
        "neumann2": HSCOptions(neumann_order=2, precision=precision),
        "schur_neumann8": HSCOptions(poly_weights=(1.0,) * NO, poly_basis="schur", precision=precision),
        "learned": HSCOptions(learned=True, precision=precision),
    }
    out = {k: {"iters": [], "pcg_ms": [], "total_ms": [], "full": [], "fallback": []} for k in modes}
    for traj in trajectories:
        ctxs = {k: HSCContext(o) for k, o in modes.items()}
        ctxs["learned"].set_learned_model(params_bf16)
        feeder = SystemFeeder(ctxs["neumann2"], traj.layout())
        for step, rows, cols, vals, meta in traj:
            ds = feeder.device_system(rows, cols, vals, traj.base.nblock, seed=traj.seed * 1000 + step)
            for k, ctx in ctxs.items():
                _, st = ctx.solve(ds, raise_on_error=False)
                out[k]["iters"].append(st["pcg_iterations"])
                out[k]["pcg_ms"].append(st["pcg_ms"])
                out[k]["total_ms"].append(st["total_ms"])
                out[k]["full"].append(st["full_relative_residual"])
                out[k]["fallback"].append(st["fallback"])
        if log:
            log(json.dumps({k: float(np.mean(v["iters"])) for k, v in out.items()}))
    return {k: {m: np.asarray(v) for m, v in d.items()} for k, d in out.items()}
