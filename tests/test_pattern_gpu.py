"""The device build of the DOF numbering, block pattern, element -> block
scatter map and element colouring (fem_dofs, fem/fem_sol.c:1263-1395;
femKhit, fem/fem_mloc.c:83-116) on meshes whose nodes and elements are
numbered at random and that hold unused nodes, against numpy statements of
the same rules:

* DOF numbers: slots 1..b of every node some element uses, numbered in node
  order (fem_dofs' slot-order numbering for one element family);
* block pattern: row I holds, sorted, every block row that shares an element
  with I;
* colouring: no two elements of one colour share a node, at most 64 colours,
  the same colours on every build;
* scatter map (indirectly): the scrambled model's solution, mapped back, is
  the unscrambled model's to round-off.

The reference's own numbering and pattern are checked bit-exact on the
golden fixtures in test_static_gpu.py.
"""
from dataclasses import replace

import numpy as np
import pytest

from ufem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def scrambled(model, seed, extra_nodes):
    """The same structure with node and element positions permuted and
    `extra_nodes` unused nodes mixed in; returns (model, node position map)."""
    rng = np.random.default_rng(seed)
    n, ne = model.nLen, model.eLen
    perm = rng.permutation(n + extra_nodes)  # old node i -> position perm[i]
    xyz = np.zeros((n + extra_nodes, 3))
    xyz[perm[:n]] = model.n_xyz
    xyz[perm[n:]] = rng.uniform(100.0, 200.0, (extra_nodes, 3))
    ep = rng.permutation(ne)
    m2 = replace(model, n_xyz=xyz, e_nodes=perm[model.e_nodes][ep], e_type=model.e_type[ep],
                 e_rs=model.e_rs[ep], e_mp=model.e_mp[ep], nl_node=perm[model.nl_node])
    return m2, perm


def expected_numbering(model):
    b = model.dofs_per_node
    used = np.zeros(model.nLen, bool)
    used[model.e_nodes.ravel()] = True
    rank = np.full(model.nLen, -1, np.int64)
    rank[used] = np.arange(used.sum())
    ndf = np.zeros((model.nLen, 7), np.int64)
    ndf[used, :b] = b * rank[used, None] + np.arange(b)[None, :] + 1
    return rank, ndf.ravel()


def expected_pattern(model, rank):
    r = rank[model.e_nodes]                       # (eLen, nn) block rows
    nn = r.shape[1]
    rows = np.repeat(r, nn, axis=1).ravel()
    cols = np.tile(r, (1, nn)).ravel()
    key = np.unique(rows * (1 << 32) + cols)
    rows, cols = key >> 32, key & 0xFFFFFFFF
    nbr = int(rank.max()) + 1
    rp = np.zeros(nbr + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp), cols


CASES = [
    ("plate", lambda: mg.plate_quad(48, 12), 101),
    ("beam", lambda: mg.beam_brick(20, 6, 6), 37),
]


@pytest.mark.parametrize("name,make,extra", CASES, ids=[c[0] for c in CASES])
def test_numbering_pattern_colouring_on_scrambled_mesh(name, make, extra):
    from ufem_b200.api import GpuModel
    base = make()
    model, _ = scrambled(base, seed=len(name), extra_nodes=extra)
    g = GpuModel(model)
    rank, ndf = expected_numbering(model)
    assert np.array_equal(g.ndoffld(model.nLen), ndf)
    assert g.ndof == model.n_active_dofs()
    rp_want, ci_want = expected_pattern(model, rank)
    rp, ci = g.bsr_pattern()
    assert np.array_equal(rp, rp_want)
    assert np.array_equal(ci, ci_want)
    col = g.element_colours()
    assert 1 <= g.colours <= 64 and col.min() == 0 and col.max() == g.colours - 1
    for c in range(g.colours):
        nodes = model.e_nodes[col == c].ravel()
        assert len(np.unique(nodes)) == len(nodes), f"colour {c} has elements sharing a node"
    g2 = GpuModel(model)
    assert np.array_equal(g2.element_colours(), col)
    g.close()
    g2.close()


@pytest.mark.parametrize("name,make,extra", CASES, ids=[c[0] for c in CASES])
def test_scrambled_mesh_solves_to_the_same_displacements(name, make, extra):
    from ufem_b200.api import GpuModel
    base = make()
    model, perm = scrambled(base, seed=len(name) + 7, extra_nodes=extra)
    b = base.dofs_per_node
    us = []
    for mdl in (base, model):
        g = GpuModel(mdl)
        rv, _ = g.fem_solve(check=False)  # assembly, supports, PCG to the reference's rule
        assert rv == 0
        ndf = g.ndoffld(mdl.nLen).reshape(-1, 7)
        u = g.u()
        us.append((ndf, u))
        g.close()
    (ndf0, u0), (ndf1, u1) = us
    a = np.stack([u0[ndf0[:, d] - 1] for d in range(b)], 1)        # base node order
    c = np.stack([u1[ndf1[perm[:base.nLen], d] - 1] for d in range(b)], 1)  # scrambled, mapped back
    assert np.abs(a - c).max() <= 1e-8 * np.abs(a).max()
