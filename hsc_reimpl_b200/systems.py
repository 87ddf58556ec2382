"""Seeded synthetic Newton systems for the HSC solve.

A system is one Newton-step Hessian of a coupled affine-body (ABD, 12 dof per
body) + FEM Tet4 (3 dof per node) model, handed to the solver the way the
libuipc global linear system hands it to ``IterativeSolver::do_solve``:

* block-COO over 3x3 blocks storing ONE triangle (row <= col), sorted by
  (row, col) with unique pairs, values column-major
  (``global_linear_system.cu:231-238`` converts to this form; the comment at
  ``linear_hsc.cu:59-60`` states the one-triangle convention; the FEM
  constitution writes ``write(min(i,j), max(i,j))`` in
  ``log_neo_hookean_3d.cu:115-131``);
* ABD dofs first, then FEM dofs (``abd_fem_linear_subsystem.cu:36-40``), so
  the layout is ``qo=0, qm=12*bodies, fo=qm, fn=3*nodes``.

Physics of the blocks (all formulas restated, none copied):

* FEM: lumped mass plus ``dt^2 V`` times the log-Neo-Hookean Hessian
  (psi = mu/2(|F|^2-3) - mu ln J + lambda/2 (ln J)^2,
  ``log_neo_hookean_function.h:77-104``), projected to SPD by clamping the
  eigenvalues of the 9x9 dPsi/dF^2 (``log_neo_hookean_function.h:106-150``)
  and pulled back with the Tet4 shape gradients.
* ABD: dyadic 12x12 mass from sample points plus the Hessian of the
  orthogonality energy kappa*V*|A A^T - I|^2 at A = I, times dt^2.
* Coupling: rank-one barrier blocks k n n^T between a FEM node and an affine
  body point (``core.py:238-248``; the 12x3 block is ``-P^T k n n^T`` with
  ``P`` the affine projection of ``core.py:201-206``), isotropic stitches for
  rim bands, and point-to-point joints between bodies.

The inputs of the workloads are synthetic: there is no public dataset.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

DT = 1.0 / 30.0


# ----------------------------------------------------------------------------
# meshes
# ----------------------------------------------------------------------------
def _orient(x, tets):
    d = np.einsum("tij->tij", x[tets[:, 1:]] - x[tets[:, :1]])
    vol = np.linalg.det(d)
    flip = vol < 0
    tets = tets.copy()
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    return tets


def cube_mesh(n=10, h=0.01):
    """n^3 cells of size h, 5 Tet4 per cell with alternating parity.

    n=10 gives 1,331 nodes and 5,000 tets.
    """
    g = np.arange(n + 1)
    I, J, K = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([I, J, K], -1).reshape(-1, 3).astype(np.float64) * h
    nid = lambda i, j, k: (i * (n + 1) + j) * (n + 1) + k
    tets = []
    even = [(0, 3, 5, 6), (1, 0, 3, 5), (2, 0, 6, 3), (4, 0, 5, 6), (7, 3, 6, 5)]
    odd = [(1, 2, 4, 7), (0, 1, 4, 2), (3, 1, 2, 7), (5, 1, 7, 4), (6, 2, 4, 7)]
    for i in range(n):
        for j in range(n):
            for k in range(n):
                c = [nid(i + (b >> 2 & 1), j + (b >> 1 & 1), k + (b & 1)) for b in range(8)]
                for t in (even if (i + j + k) % 2 == 0 else odd):
                    tets.append([c[t[0]], c[t[1]], c[t[2]], c[t[3]]])
    tets = np.asarray(tets, dtype=np.int64)
    return x, _orient(x, tets)


def annulus_mesh(r_in=0.27, r_out=0.47, width=0.3, nr=4, na=5, nc=93, center=(0.0, 0.0, 0.0)):
    """Tet4 annulus (a tire torus of rectangular section), Kuhn 6-tet split.

    Node (ir, ia, ic) sits at radius r_in + ir*dr, axial offset
    -width/2 + ia*da, angle 2*pi*ic/nc; the ring is periodic in ic.
    nr=4, na=5, nc=93 gives 2,790 nodes and 11,160 tets per tire.
    """
    r = np.linspace(r_in, r_out, nr + 1)
    a = np.linspace(-width / 2, width / 2, na + 1)
    th = 2 * np.pi * np.arange(nc) / nc
    R, A, T = np.meshgrid(r, a, th, indexing="ij")
    x = np.stack([R * np.cos(T), A, R * np.sin(T)], -1).reshape(-1, 3) + np.asarray(center)
    nid = lambda ir, ia, ic: (ir * (na + 1) + ia) * nc + (ic % nc)
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    ir, ia, ic = np.meshgrid(np.arange(nr), np.arange(na), np.arange(nc), indexing="ij")
    ir, ia, ic = ir.ravel(), ia.ravel(), ic.ravel()
    tets = []
    for p in perms:
        cur = np.zeros((3, ir.size), dtype=np.int64)
        verts = [nid(ir, ia, ic)]
        for axis in p:
            cur[axis] += 1
            verts.append(nid(ir + cur[0], ia + cur[1], ic + cur[2]))
        tets.append(np.stack(verts, -1))
    tets = np.concatenate(tets, 0)
    grid = dict(nr=nr, na=na, nc=nc)
    return x, _orient(x, tets), grid


# ----------------------------------------------------------------------------
# log-Neo-Hookean FEM Hessian
# ----------------------------------------------------------------------------
def lame(E, nu):
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


def _cofactor(F):
    C = np.empty_like(F)
    for i in range(3):
        for j in range(3):
            C[:, i, j] = (F[:, (i + 1) % 3, (j + 1) % 3] * F[:, (i + 2) % 3, (j + 2) % 3]
                          - F[:, (i + 1) % 3, (j + 2) % 3] * F[:, (i + 2) % 3, (j + 1) % 3])
    return C


def log_nh_dPdF(F, mu, lam, project=True):
    """9x9 Hessian d^2 psi / dvec(F)^2 of log-NH, column-major vec(F).

    H[i+3a, j+3b] = mu d_ij d_ab + lam G_ia G_jb - (lam ln J - mu) G_ib G_ja,
    G = cof(F)/J; then eigenvalues are clamped at 0 when ``project``.
    """
    T = F.shape[0]
    J = np.linalg.det(F)
    G = _cofactor(F) / J[:, None, None]
    q = lam * np.log(J) - mu
    mu = np.broadcast_to(np.asarray(mu, dtype=np.float64), (T,))
    lam = np.broadcast_to(np.asarray(lam, dtype=np.float64), (T,))
    H = lam[:, None, None, None, None] * np.einsum("tia,tjb->taibj", G, G)
    H -= q[:, None, None, None, None] * np.einsum("tib,tja->taibj", G, G)
    H = H.reshape(T, 9, 9)
    H += mu[:, None, None] * np.eye(9)
    if project:
        w, Q = np.linalg.eigh(H)
        H = np.einsum("tik,tk,tjk->tij", Q, np.maximum(w, 0.0), Q)
    return H


def fem_hessian(x_rest, tets, E, nu, rho, dt=DT, perturb=0.0, rng=None):
    """Lumped mass + dt^2 V log-NH Hessian (SPD-projected) as COO triplets."""
    nn = x_rest.shape[0]
    Dm = np.transpose(x_rest[tets[:, 1:]] - x_rest[tets[:, :1]], (0, 2, 1))  # columns = edges
    vol = np.abs(np.linalg.det(Dm)) / 6.0
    Dminv = np.linalg.inv(Dm)
    x = x_rest
    if perturb > 0:
        h = np.cbrt(vol.mean())
        x = x_rest + perturb * h * rng.standard_normal(x_rest.shape)
    Ds = np.transpose(x[tets[:, 1:]] - x[tets[:, :1]], (0, 2, 1))
    F = Ds @ Dminv
    E = np.broadcast_to(np.asarray(E, dtype=np.float64), (tets.shape[0],))
    mu, lam = lame(E, nu)
    # shape gradients: F[i,a] = sum_k x_k[i] Gs[k,a]
    Gs = np.concatenate([-Dminv.sum(1, keepdims=True), Dminv], 1)  # (T,4,3)
    rows, cols, vals = [], [], []
    chunk = 65536
    li = np.arange(12)
    for s in range(0, tets.shape[0], chunk):
        e = slice(s, s + chunk)
        H9 = log_nh_dPdF(F[e], mu[e], lam[e], project=perturb > 0).reshape(-1, 3, 3, 3, 3)  # t,a,i,b,j
        Ke = np.einsum("tka,tlb,taibj->tkilj", Gs[e], Gs[e], H9)
        Ke *= (vol[e] * dt * dt)[:, None, None, None, None]
        dof = (3 * tets[e][:, :, None] + np.arange(3)).reshape(-1, 12)
        rows.append(np.repeat(dof, 12, axis=1).ravel())
        cols.append(np.tile(dof, (1, 12)).ravel())
        vals.append(Ke.reshape(-1, 144).ravel())
    node_mass = np.zeros(nn)
    np.add.at(node_mass, tets.ravel(), np.repeat(rho * vol / 4.0, 4))
    d = np.arange(3 * nn)
    rows.append(d)
    cols.append(d)
    vals.append(np.repeat(node_mass, 3))
    return np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), node_mass


# ----------------------------------------------------------------------------
# affine bodies
# ----------------------------------------------------------------------------
def affine_projection(rest):
    """3x12 map q -> x for dof order [A row0, A row1, A row2, p] (core.py:201-206)."""
    P = np.zeros((3, 12))
    for r in range(3):
        P[r, 3 * r:3 * r + 3] = rest
        P[r, 9 + r] = 1.0
    return P


def abd_block(mass, points, kappa, volume, dt=DT):
    """Dyadic mass over sample points plus dt^2 * Hessian of kappa V |A A^T - I|^2 at A=I."""
    M = np.zeros((12, 12))
    w = mass / len(points)
    for p in points:
        P = affine_projection(p)
        M += w * P.T @ P
    S = np.zeros((9, 9))  # vec(dA) -> vec(dA + dA^T), row-major A
    for i in range(3):
        for j in range(3):
            S[3 * i + j, 3 * i + j] += 1
            S[3 * i + j, 3 * j + i] += 1
    M[:9, :9] += dt * dt * 2.0 * kappa * volume * (S.T @ S)
    return M


@dataclass
class HSCSystem:
    """One Newton-step linear system in the solver's input form."""
    name: str
    layout: tuple            # (qo, qm, fo, fn)
    H: sp.csr_matrix         # full symmetric matrix, N x N
    rows: np.ndarray         # int32 block rows, one triangle, sorted, unique
    cols: np.ndarray         # int32 block cols
    vals: np.ndarray         # float64 (nnzb, 3, 3) block values (row-major in numpy)
    b: np.ndarray
    x_star: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def N(self):
        return self.H.shape[0]

    @property
    def nblock(self):
        return self.H.shape[0] // 3

    def values_colmajor(self):
        """(nnzb, 9) with element (r, c) at r + 3c, as Eigen Matrix3x3 stores it."""
        return np.ascontiguousarray(np.transpose(self.vals, (0, 2, 1)).reshape(-1, 9))


def bcoo_upper_from_csr(H):
    """One-triangle (row <= col) sorted unique 3x3 BCOO of a symmetric CSR matrix."""
    B = sp.csr_matrix(H).tobsr(blocksize=(3, 3))
    B.sort_indices()
    nbr = B.shape[0] // 3
    brow = np.repeat(np.arange(nbr), np.diff(B.indptr))
    bcol = B.indices
    keep = bcol >= brow
    return (brow[keep].astype(np.int32), bcol[keep].astype(np.int32),
            np.ascontiguousarray(B.data[keep], dtype=np.float64))


class _Assembler:
    def __init__(self, N):
        self.N = N
        self.r, self.c, self.v = [], [], []

    def add(self, rows, cols, vals):
        self.r.append(np.asarray(rows, dtype=np.int64).ravel())
        self.c.append(np.asarray(cols, dtype=np.int64).ravel())
        self.v.append(np.asarray(vals, dtype=np.float64).ravel())

    def add_dense(self, dofs, M):
        dofs = np.asarray(dofs)
        self.add(np.repeat(dofs, len(dofs)), np.tile(dofs, len(dofs)), M)

    def add_outer(self, dofs, g, k):
        """H += k g g^T on the listed dofs (g dense over dofs)."""
        self.add_dense(dofs, k * np.outer(g, g))

    def csr(self):
        H = sp.coo_matrix((np.concatenate(self.v), (np.concatenate(self.r), np.concatenate(self.c))),
                          shape=(self.N, self.N)).tocsr()
        H.sum_duplicates()
        H.eliminate_zeros()
        return H


def _finish(name, asm, layout, rng, meta):
    H = asm.csr()
    H = ((H + H.T) * 0.5).tocsr()
    rows, cols, vals = bcoo_upper_from_csr(H)
    x_star = rng.standard_normal(H.shape[0])
    b = H @ x_star
    s = np.linalg.norm(b)
    meta = dict(meta)
    meta.update(nnzb=int(rows.size), N=int(H.shape[0]))
    return HSCSystem(name, layout, H, rows, cols, vals, b / s, x_star / s, meta)


def _barrier_coupling(asm, qm, node, body, rest, normal, k):
    """Rank-one contact between FEM node and affine body point (core.py:238-248 form)."""
    P = affine_projection(rest)
    dofs = np.concatenate([qm + 3 * node + np.arange(3), 12 * body + np.arange(12)])
    g = np.concatenate([normal, -normal @ P])
    asm.add_outer(dofs, g, k)


def _stitch(asm, qm, node, body, rest, k):
    for axis in range(3):
        n = np.zeros(3)
        n[axis] = 1.0
        _barrier_coupling(asm, qm, node, body, rest, n, k)


def _joint(asm, body_a, pa, body_b, pb, k):
    Pa, Pb = affine_projection(pa), affine_projection(pb)
    dofs = np.concatenate([12 * body_a + np.arange(12), 12 * body_b + np.arange(12)])
    for axis in range(3):
        g = np.concatenate([Pa[axis], -Pb[axis]])
        asm.add_outer(dofs, g, k)


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------
def make_cube_system(seed=0, n=10, h=0.01, E=1e6, nu=0.45, rho=1000.0, E_abd=1e10,
                     k_range=(1e6, 1e9), perturb=0.02):
    """One ABD plate under a 10x10x10-cell Tet4 cube (1,331 nodes, 5,000 tets).

    The 121 bottom-face nodes touch the plate through barrier blocks with
    stiffness log-uniform in ``k_range``; contact normals are +z tilted by a
    seeded 10 % jitter.
    """
    rng = np.random.default_rng(seed)
    x, tets = cube_mesh(n, h)
    nn = x.shape[0]
    qm, fn = 12, 3 * nn
    asm = _Assembler(qm + fn)
    r, c, v, node_mass = fem_hessian(x, tets, E, nu, rho, perturb=perturb, rng=rng)
    asm.add(qm + r, qm + c, v)
    bottom = np.flatnonzero(np.isclose(x[:, 2], 0.0))
    center = np.array([n * h / 2, n * h / 2, -h])
    plate_pts = x[bottom] - center
    plate_vol = (n * h) ** 2 * h
    asm.add_dense(np.arange(12), abd_block(rho * plate_vol, plate_pts, E_abd, plate_vol))
    ks = np.exp(rng.uniform(np.log(k_range[0]), np.log(k_range[1]), bottom.size))
    for node, k in zip(bottom, ks):
        nrm = np.array([0.0, 0.0, 1.0]) + 0.1 * rng.standard_normal(3)
        nrm /= np.linalg.norm(nrm)
        _barrier_coupling(asm, qm, node, 0, x[node] - center, nrm, k)
    meta = dict(config="cube", nodes=nn, tets=int(tets.shape[0]), bodies=1,
                coupled_nodes=int(bottom.size), seed=seed)
    return _finish("cube_1331", asm, (0, qm, qm, fn), rng, meta)


def make_vehicle_system(seed=0, nr=4, na=5, nc=93, E_carried=1e10, E_ground=1e6, nu=0.3,
                        rho=1000.0, E_abd=1e10, contact_frac=(0.05, 0.15),
                        k_range=(1e6, 1e9), k_rim=1e7, k_joint=1e9, perturb=0.02):
    """Vehicle-scale system: 7 Tet4 tire tori + 12 affine bodies.

    Tires 0-3 are carried (E=1e10), 4-6 lie on the ground (E=1e6). Bodies
    0-6 are the rims (one per tire, stitched to 38 rim-band nodes), 7-10 are
    spindles jointed to rims 0-3 and to each other, 11 is the ground body
    that every tire's contact patch (5-15 % of its tread nodes) touches.
    """
    rng = np.random.default_rng(seed)
    ntire, nbody = 7, 12
    meshes = []
    for t in range(ntire):
        center = np.array([1.2 * (t % 4), 0.5 * (t // 4), 0.0])
        x, tets, grid = annulus_mesh(nr=nr, na=na, nc=nc, center=center)
        meshes.append((x, tets, center))
    nodes_per = meshes[0][0].shape[0]
    nn = ntire * nodes_per
    qm, fn = 12 * nbody, 3 * nn
    asm = _Assembler(qm + fn)
    ntets = 0
    active_nodes = 0
    for t, (x, tets, center) in enumerate(meshes):
        base = t * nodes_per
        E = E_carried if t < 4 else E_ground
        r, c, v, _ = fem_hessian(x, tets, E, nu, rho, perturb=perturb, rng=rng)
        asm.add(qm + 3 * base + r, qm + 3 * base + c, v)
        ntets += tets.shape[0]
        # rim band: inner-surface nodes on both axial edges, every 5th station
        rim = [((0 * (na + 1) + ia) * nc + ic) for ia in (0, na) for ic in range(0, nc, 5)]
        rim_pts = x[rim] - center
        rim_vol = np.pi * 0.27 ** 2 * 0.3 * 0.1
        asm.add_dense(12 * t + np.arange(12), abd_block(20.0, rim_pts, E_abd, rim_vol))
        for node in rim:
            _stitch(asm, qm, base + node, t, x[node] - center, k_rim)
        active_nodes += len(rim)
        # contact patch on the tread (outer surface), centred at a seeded angle
        tread = np.array([((nr * (na + 1) + ia) * nc + ic) for ia in range(na + 1) for ic in range(nc)])
        frac = rng.uniform(*contact_frac)
        count = max(1, int(round(frac * tread.size)))
        th0 = rng.uniform(0, 2 * np.pi)
        ang = np.arctan2(x[tread, 2] - center[2], x[tread, 0] - center[0])
        dist = np.abs(np.angle(np.exp(1j * (ang - th0))))
        patch = tread[np.argsort(dist, kind="stable")[:count]]
        ks = np.exp(rng.uniform(np.log(k_range[0]), np.log(k_range[1]), patch.size))
        for node, k in zip(patch, ks):
            nrm = x[node] - center
            nrm[1] = 0.0
            nrm /= np.linalg.norm(nrm)
            nrm += 0.05 * rng.standard_normal(3)
            nrm /= np.linalg.norm(nrm)
            _barrier_coupling(asm, qm, base + node, 11, x[node] - np.array([1.8, 0.25, -1.0]), nrm, k)
        active_nodes += patch.size
    for s in range(4):  # spindles
        pts = rng.uniform(-0.1, 0.1, (16, 3))
        asm.add_dense(12 * (7 + s) + np.arange(12), abd_block(10.0, pts, E_abd, 0.004))
        for p in (np.array([0.0, 0.1, 0.0]), np.array([0.05, 0.1, 0.05]), np.array([0.0, 0.1, 0.08])):
            _joint(asm, 7 + s, p, s, p + np.array([0.0, -0.25, 0.0]), k_joint)
    for s in range(3):
        _joint(asm, 7 + s, np.array([0.3, 0.0, 0.0]), 8 + s, np.array([-0.3, 0.0, 0.0]), 1e-2 * k_joint)
    gpts = rng.uniform(-2.0, 2.0, (32, 3))
    asm.add_dense(12 * 11 + np.arange(12), abd_block(1e4, gpts, E_abd, 10.0))
    meta = dict(config="vehicle", nodes=nn, tets=ntets, bodies=nbody, tires=ntire,
                coupled_nodes=int(active_nodes), seed=seed)
    return _finish("vehicle_7tires", asm, (0, qm, qm, fn), rng, meta)


def tire_mesh():
    """The vehicle scene's Tet4 tire (3,548 nodes, 11,171 tets, tire axis = local y) and
    the placements of the seven tires the vehicle workload uses (four mounted, three
    lying flat), as extracted by ``hsc_reimpl_b200/data/make_tire_mesh.py``."""
    from pathlib import Path
    return np.load(Path(__file__).resolve().parent / "data" / "tire_tet4.npz")


def make_reference_vehicle_system(seed=0, E_carried=1e10, E_ground=1e6, nu=0.3, rho=1000.0,
                                  E_abd=1e10, contact_frac=(0.05, 0.15), k_range=(1e6, 1e9),
                                  k_rim=1e7, k_joint=1e9, perturb=0.02, tread_radius=0.4259):
    """Vehicle-scale system on the vehicle scene's own tire mesh: 7 tires x 3,548 nodes =
    24,836 nodes (74,508 FEM dofs), 78,197 Tet4, 149,513 upper blocks, 12 affine bodies.

    Tires 0-3 are the mounted (carried) tires, E = ``E_carried``; 4-6 lie on the ground,
    E = ``E_ground``; positions and orientations are the scene's.  Bodies 0-6 are the
    rims, each stitched to its tire's 39 rim-connection nodes (``BC_CONN``); 7-10 are
    spindles jointed to rims 0-3 and to each other; 11 is the ground body.  Each tire's
    contact patch is the seeded share ``contact_frac`` of its tread-node count (surface
    nodes at tire radius >= ``tread_radius``), taken as the surface nodes nearest the
    ground plane z = 0; each patch node touches the ground body through a barrier block
    k n n^T, k log-uniform in ``k_range``, n = +z with a 5 % seeded tilt.
    """
    rng = np.random.default_rng(seed)
    m = tire_mesh()
    xl, tl = m["vertices"], m["tetrahedra"].astype(np.int64)
    conn = m["bc_conn"].astype(np.int64)
    surf = np.unique(m["surface_triangles"])
    rad = np.hypot(xl[:, 0], xl[:, 2])
    ntread = int(np.count_nonzero(rad[surf] >= tread_radius))
    Rs, Ts, mounted = m["placement_rotation"], m["placement_translation"], m["placement_mounted"]
    ntire, nbody = Rs.shape[0], 12
    nodes_per = xl.shape[0]
    nn = ntire * nodes_per
    qm, fn = 12 * nbody, 3 * nn
    asm = _Assembler(qm + fn)
    ground_center = np.array([-1.5, 0.0, -1.0])
    ntets = active_nodes = 0
    for t in range(ntire):
        x = xl @ Rs[t].T + Ts[t]
        tets = _orient(x, tl)
        center = Ts[t]
        base = t * nodes_per
        E = E_carried if mounted[t] else E_ground
        r, c, v, _ = fem_hessian(x, tets, E, nu, rho, perturb=perturb, rng=rng)
        asm.add(qm + 3 * base + r, qm + 3 * base + c, v)
        ntets += tets.shape[0]
        rim_pts = x[conn] - center
        rim_vol = np.pi * 0.25 ** 2 * 0.28 * 0.1
        asm.add_dense(12 * t + np.arange(12), abd_block(20.0, rim_pts, E_abd, rim_vol))
        for node in conn:
            _stitch(asm, qm, base + node, t, x[node] - center, k_rim)
        active_nodes += conn.size
        frac = rng.uniform(*contact_frac)
        count = max(1, int(round(frac * ntread)))
        cand = surf[~np.isin(surf, conn)]
        patch = cand[np.argsort(x[cand, 2], kind="stable")[:count]]
        ks = np.exp(rng.uniform(np.log(k_range[0]), np.log(k_range[1]), patch.size))
        for node, k in zip(patch, ks):
            nrm = np.array([0.0, 0.0, 1.0]) + 0.05 * rng.standard_normal(3)
            nrm /= np.linalg.norm(nrm)
            _barrier_coupling(asm, qm, base + node, 11, x[node] - ground_center, nrm, k)
        active_nodes += patch.size
    for s in range(4):  # spindles
        pts = rng.uniform(-0.1, 0.1, (16, 3))
        asm.add_dense(12 * (7 + s) + np.arange(12), abd_block(10.0, pts, E_abd, 0.004))
        for p in (np.array([0.0, 0.1, 0.0]), np.array([0.05, 0.1, 0.05]), np.array([0.0, 0.1, 0.08])):
            _joint(asm, 7 + s, p, s, p + np.array([0.0, -0.25, 0.0]), k_joint)
    for s in range(3):
        _joint(asm, 7 + s, np.array([0.3, 0.0, 0.0]), 8 + s, np.array([-0.3, 0.0, 0.0]), 1e-2 * k_joint)
    gpts = rng.uniform(-2.0, 2.0, (32, 3))
    asm.add_dense(12 * 11 + np.arange(12), abd_block(1e4, gpts, E_abd, 10.0))
    meta = dict(config="vehicle_tire_tet4", nodes=nn, tets=ntets, bodies=nbody, tires=ntire,
                coupled_nodes=int(active_nodes), seed=seed, mesh="tire_tet4")
    return _finish("vehicle_tire_tet4_78k", asm, (0, qm, qm, fn), rng, meta)


def make_torus_system(seed=0, target_tets=10000, bodies=4, E=1e8, nu=0.3, rho=1000.0,
                      E_abd=1e10, contact_frac=0.1, k_range=(1e6, 1e9), k_rim=1e7,
                      nr=3, na=4, E_rim=None, perturb=0.02, name="torus"):
    """One tire torus with ``bodies`` affine bodies: rim segments (all but the
    last body, each stitched to an arc of the inner surface) and a ground body
    touched by a ``contact_frac`` share of the tread nodes.
    ``E_rim`` (if set) is the modulus of the innermost radial cell layer.
    """
    rng = np.random.default_rng(seed)
    nc = max(8, int(round(target_tets / (6 * nr * na))))
    x, tets, grid = annulus_mesh(nr=nr, na=na, nc=nc)
    nn = x.shape[0]
    qm, fn = 12 * bodies, 3 * nn
    asm = _Assembler(qm + fn)
    Et = np.full(tets.shape[0], float(E))
    if E_rim is not None:
        rad = np.linalg.norm(x[tets][:, :, [0, 2]], axis=2).mean(1)
        Et[rad < 0.27 + (0.47 - 0.27) / nr] = E_rim
    r, c, v, _ = fem_hessian(x, tets, Et, nu, rho, perturb=perturb, rng=rng)
    asm.add(qm + r, qm + c, v)
    nrim = max(1, bodies - 1)
    inner = np.array([(ia * nc + ic) for ia in (0, na) for ic in range(nc)])
    ang = np.arctan2(x[inner, 2], x[inner, 0]) % (2 * np.pi)
    seg = np.minimum((ang / (2 * np.pi) * nrim).astype(int), nrim - 1)
    active = 0
    for bidx in range(nrim):
        sel = inner[seg == bidx][::2]
        c0 = x[sel].mean(0)
        asm.add_dense(12 * bidx + np.arange(12), abd_block(5.0, x[sel] - c0, E_abd, 0.01))
        for node in sel:
            _stitch(asm, qm, node, bidx, x[node] - c0, k_rim)
        active += sel.size
    if bodies >= 2:
        gb = bodies - 1
        gpts = rng.uniform(-2.0, 2.0, (32, 3))
        asm.add_dense(12 * gb + np.arange(12), abd_block(1e4, gpts, E_abd, 10.0))
        tread = np.array([((nr * (na + 1) + ia) * nc + ic) for ia in range(na + 1) for ic in range(nc)])
        count = max(1, int(round(contact_frac * tread.size)))
        th0 = rng.uniform(0, 2 * np.pi)
        angt = np.arctan2(x[tread, 2], x[tread, 0])
        patch = tread[np.argsort(np.abs(np.angle(np.exp(1j * (angt - th0)))), kind="stable")[:count]]
        ks = np.exp(rng.uniform(np.log(k_range[0]), np.log(k_range[1]), patch.size))
        for node, k in zip(patch, ks):
            nrm = x[node].copy()
            nrm[1] = 0.0
            nrm /= np.linalg.norm(nrm)
            _barrier_coupling(asm, qm, node, gb, x[node] - np.array([0.0, 0.0, -1.0]), nrm, k)
        active += patch.size
        for bidx in range(min(nrim, gb)):
            if bidx + 1 < nrim:
                _joint(asm, bidx, np.array([0.1, 0.0, 0.0]), bidx + 1, np.array([-0.1, 0.0, 0.0]), 1e8)
    meta = dict(config=name, nodes=nn, tets=int(tets.shape[0]), bodies=bodies,
                coupled_nodes=int(active), seed=seed)
    return _finish(name, asm, (0, qm, qm, fn), rng, meta)


def make_stress_system(seed=0, target_tets=1_000_000, contact_frac=0.30, perturb=0.0):
    """One torus refined to ~1.0 M Tet4 (nr=8, na=12), 12 affine bodies,
    E=1e10 rim layer against a 1e6 Pa tread, 30 % contact-active tread nodes.
    ``perturb=0`` assembles at rest, where the log-NH Hessian is already PSD.
    """
    return make_torus_system(seed=seed, target_tets=target_tets, bodies=12, E=1e6, E_rim=1e10,
                             contact_frac=contact_frac, nr=8, na=12, perturb=perturb,
                             name="stress_torus_1M")


def make_batch_systems(seed=0, count=64, tet_range=(2000, 40000), body_range=(1, 12),
                       E_range=(1e6, 1e10)):
    """Uneven systems: tets log-uniform in ``tet_range``, cube or torus meshes,
    1-12 affine bodies, E log-uniform in ``E_range``."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        T = float(np.exp(rng.uniform(np.log(tet_range[0]), np.log(tet_range[1]))))
        nb = int(rng.integers(body_range[0], body_range[1] + 1))
        E = float(np.exp(rng.uniform(np.log(E_range[0]), np.log(E_range[1]))))
        s = int(rng.integers(1 << 30))
        if rng.uniform() < 0.5 and nb == 1:
            n = max(3, int(round((T / 5) ** (1 / 3))))
            sysm = make_cube_system(seed=s, n=n, h=0.1 / n, E=E)
        else:
            sysm = make_torus_system(seed=s, target_tets=T, bodies=max(nb, 1), E=E, name="torus")
        sysm.meta["batch_index"] = i
        out.append(sysm)
    return out


def from_dense_fixture(D, A, E, b):
    """Wrap a dense (D, A, E) fixture in the solver input form.

    The fixture order is FEM first then ABD (H = [[D, E^T], [E, A]]), so the
    layout is ``fo=0, fn=len(D), qo=len(D), qm=len(A)``.
    """
    n, m = D.shape[0], A.shape[0]
    H = np.zeros((n + m, n + m))
    H[:n, :n], H[n:, n:], H[n:, :n], H[:n, n:] = D, A, E, E.T
    Hs = sp.csr_matrix(H)
    rows, cols, vals = bcoo_upper_from_csr(Hs)
    return HSCSystem("fixture", (n, m, 0, n), Hs, rows, cols, vals, np.asarray(b, dtype=np.float64),
                     np.zeros(n + m), dict(config="fixture", N=n + m, nnzb=int(rows.size)))
