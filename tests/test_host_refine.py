"""Host logic of exf_mesh_refine_arrays (no GPU): uniform refinement of a coarse quad9 /
hex27 mesh into a level-nested hierarchy, checked against the oracle's structured
hierarchy of the same box, for nesting, neighbours and parents, and on a curved coarse
mesh against the element map evaluated here."""
import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib

ABC2 = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]


def rows(a):
    """Rows of a [n][k] array in lexicographic order (rounded to 1e-12)."""
    a = np.round(np.asarray(a, float), 12)
    return a[np.lexsort(a.T[::-1])]


def box_case(oracle_mod, dim, nlev, n0, box):
    om = oracle_mod.OrMesh(dim, nlev, n0, box)
    c0, _, _ = om.conn(0)
    r = ex.Mesh.refine_arrays(dim, nlev, om.nvert0, om.xyz()[:, :om.nnodes(0)], c0)
    return om, r


CASES = [(2, 4, (2, 3), (0, 2, 0, 1)), (3, 3, (2, 1, 2), (0, 2, 0, 1, 0, 1))]


@pytest.mark.parametrize("dim,nlev,n0,box", CASES)
def test_refined_box_equals_structured_hierarchy(oracle_mod, dim, nlev, n0, box):
    om, r = box_case(oracle_mod, dim, nlev, n0, box)
    X = om.xyz()
    for lev in range(nlev):
        assert r["nnodes"][lev] == om.nnodes(lev) and r["nel"][lev] == om.nel(lev)
        # the same points, and the same elements as point sets (centroids)
        assert np.array_equal(rows(r["xyz"][:, :r["nnodes"][lev]].T), rows(X[:, :om.nnodes(lev)].T))
        oc, onb, _ = om.conn(lev)
        cg = r["xyz"][:, r["conn"][lev]].mean(axis=2).T
        co = X[:, oc].mean(axis=2).T
        assert np.array_equal(rows(cg), rows(co))
        assert (r["neigh"][lev] < 0).sum() == (onb < 0).sum()  # boundary sides


@pytest.mark.parametrize("dim,nlev,n0,box", CASES)
def test_nesting_neighbours_and_parents(oracle_mod, dim, nlev, n0, box):
    """Level-nested numbering (vertices of level L are the nodes of level L-1, the other
    element nodes new), symmetric neighbours, and each child a sub-cell of its parent that
    shares the parent's vertex at its own corner."""
    om, r = box_case(oracle_mod, dim, nlev, n0, box)
    nvx = 4 if dim == 2 else 8
    X = r["xyz"]
    for lev in range(nlev):
        c, nb = r["conn"][lev], r["neigh"][lev]
        below = om.nvert0 if lev == 0 else r["nnodes"][lev - 1]
        assert np.all(c[:, :nvx] < below) and np.all(c[:, nvx:] >= below)
        assert np.all(c < r["nnodes"][lev])
        for e in range(c.shape[0]):
            for f in nb[e]:
                if f >= 0:
                    assert e in nb[f]
        if lev == 0:
            continue
        par = r["parent"][lev]
        pc = r["conn"][lev - 1]
        assert np.array_equal(np.bincount(par, minlength=pc.shape[0]), np.full(pc.shape[0], 2 ** dim))
        for e in range(c.shape[0]):
            p = pc[par[e]]
            shared = [k for k in range(nvx) if c[e, k] == p[k]]
            assert len(shared) == 1  # the child's corner vertex is the parent's
            lo, hi = X[:, p].min(axis=1)[:, None], X[:, p].max(axis=1)[:, None]
            assert np.all(X[:, c[e]] >= lo - 1e-12) and np.all(X[:, c[e]] <= hi + 1e-12)


def lag(a, s):
    return (0.5 * s * (s - 1.0), 1.0 - s * s, 0.5 * s * (s + 1.0))[a]


def test_curved_coarse_mesh_keeps_the_element_map():
    """A quarter annulus of two quad9 elements whose edge and centre nodes lie on the arcs:
    every new node is the biquadratic map of its parent at the node's reference point."""
    r0, r1 = 1.0, 2.0
    # vertices first: (r, theta) grid 2 x 3 vertices, then mid-edge and centre nodes
    pts, index = [], {}

    def node(i, j):  # i: radial offset 0..2, j: angular offset 0..4 (half-element units)
        if (i, j) not in index:
            rr = r0 + (r1 - r0) * i / 2.0
            th = 0.5 * np.pi * j / 4.0
            index[(i, j)] = len(pts)
            pts.append((rr * np.cos(th), rr * np.sin(th)))
        return index[(i, j)]

    for i in (0, 2):
        for j in (0, 2, 4):
            node(i, j)
    nvert0 = len(pts)
    conn = []
    for e in range(2):
        conn.append([node(a, 2 * e + b) for a, b in ABC2])
    xyz0 = np.array(pts).T
    r = ex.Mesh.refine_arrays(2, 3, nvert0, xyz0, np.array(conn))
    X = r["xyz"]
    for lev in (1, 2):
        pc = r["conn"][lev - 1]
        for e, ce in enumerate(r["conn"][lev]):
            p = pc[r["parent"][lev][e]]
            ch = e % 4
            cx, cy = ch & 1, ch >> 1
            for k, (a, b) in enumerate(ABC2):
                s, t = 0.5 * (2 * cx + a) - 1.0, 0.5 * (2 * cy + b) - 1.0
                w = np.array([lag(aa, s) * lag(bb, t) for aa, bb in ABC2])
                assert np.abs(X[:, p] @ w - X[:, ce[k]]).max() < 1e-14
    # the new level-1 points on the outer arc stay close to it (quadratic arcs)
    rad = np.hypot(X[0], X[1])
    assert np.all(rad > r0 - 1e-3) and np.all(rad < r1 + 1e-3)


def test_bad_coarse_mesh_is_refused():
    xyz0 = np.array([[0, 1, 1, 0, 0.5, 1, 0.5, 0, 0.5], [0, 0, 1, 1, 0, 0.5, 1, 0.5, 0.5]], float)
    conn = np.arange(9)[None, :]
    r = ex.Mesh.refine_arrays(2, 2, 4, xyz0, conn)
    assert list(r["nnodes"]) == [9, 25]
    bad = conn.copy()
    bad[0, [0, 4]] = bad[0, [4, 0]]  # a mid-edge node where a vertex belongs
    with pytest.raises(_lib.ExfError) as e:
        ex.Mesh.refine_arrays(2, 2, 4, xyz0, bad)
    assert e.value.code == _lib.EXF_ERR_ARG
