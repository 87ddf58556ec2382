"""The FEM node partition of the analysis (hsc_partition.cpp), called on the host.

The persistent PCG gives each CTA one part as a contiguous row range, so the
parts must cover every node once, be balanced in weight (a CTA's work) and be
compact (few blocks reach other parts: small vector windows, and a block-local
preconditioner that captures most of D).  Deterministic: the same input gives the
same parts.
"""
import numpy as np
import scipy.sparse as sp

from hsc_reimpl_b200 import _lib


def _graph(s):
    fb0 = s.layout[2] // 3
    m = (s.rows >= fb0) & (s.cols >= fb0) & (s.rows != s.cols)
    r, c = s.rows[m] - fb0, s.cols[m] - fb0
    n = s.layout[3] // 3
    G = sp.csr_matrix((np.ones(2 * r.size), (np.r_[r, c], np.r_[c, r])), shape=(n, n))
    G.sort_indices()
    return G


def _partition(G, w, P):
    lib = _lib.load()
    part = np.zeros(G.shape[0], dtype=np.int32)
    ptr = np.ascontiguousarray(G.indptr, dtype=np.int32)
    adj = np.ascontiguousarray(G.indices, dtype=np.int32)
    w = np.ascontiguousarray(w, dtype=np.float64)
    rc = lib.hsc_partition_nodes(G.shape[0], ptr.ctypes.data, adj.ctypes.data, w.ctypes.data, P, part.ctypes.data)
    assert rc == _lib.HSC_OK
    return part


def test_tire_mesh_partition_is_balanced_and_compact():
    from hsc_reimpl_b200.systems import make_reference_vehicle_system
    s = make_reference_vehicle_system(seed=0)
    G = _graph(s)
    deg = np.diff(G.indptr)
    w = 2.0 + deg                      # the analysis' weight: 1 + blocks of the row (diagonal included)
    part = _partition(G, w, 148)
    assert part.min() == 0 and part.max() == 147
    load = np.bincount(part, weights=w, minlength=148)
    assert load.max() <= 1.1 * load.mean(), (load.min(), load.max(), load.mean())
    rows = np.repeat(np.arange(G.shape[0]), deg)
    cross = np.mean(part[rows] != part[G.indices])
    # the mesh's own numbering cut into 148 equal ranges crosses parts on most edges
    natural = np.minimum(np.arange(G.shape[0]) * 148 // G.shape[0], 147)
    cross_nat = np.mean(natural[rows] != natural[G.indices])
    assert cross < 0.2 and cross < 0.3 * cross_nat, (cross, cross_nat)
    np.testing.assert_array_equal(part, _partition(G, w, 148))


def test_partition_of_disconnected_components_and_tiny_inputs():
    # two disjoint paths of 10 nodes: 4 parts, two per path, contiguous along the path
    n = 20
    r = np.r_[np.arange(9), np.arange(10, 19)]
    G = sp.csr_matrix((np.ones(2 * r.size), (np.r_[r, r + 1], np.r_[r + 1, r])), shape=(n, n))
    G.sort_indices()
    part = _partition(G, np.ones(n), 4)
    assert set(part[:10]) & set(part[10:]) == set()
    assert np.bincount(part).tolist() == [5, 5, 5, 5]
    for p in range(4):
        idx = np.flatnonzero(part == p)
        assert idx.max() - idx.min() == idx.size - 1       # a contiguous piece of its path
    assert _partition(G, np.ones(n), 1).tolist() == [0] * n
