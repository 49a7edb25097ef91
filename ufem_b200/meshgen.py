"""Structured meshes and uFEM input files for the linear static path.

Every model is held in the same flat tables the reference reader fills
(``femReadInput``, fem/fem_io.c:380-590): node coordinates ``n_x/n_y/n_z``;
element type, real set, material and node lists (``eType/eRS/eMP/eFrom/
eNodesL``); real sets and materials as (type, value list); nodal loads and
supports ``nlNode/nlType/nlDir/nlVal``.  All positions are 0-based, which is
the reference's "preparsed" input variant (fem/feminput.5, "(P)" fields;
``femRenumIndex`` returns at once for it, fem/fem_io.c:55).

Node numbering is lexicographic with x fastest.  Element node order follows the
reference's natural coordinates: the quad goes (-1,-1),(1,-1),(1,1),(-1,1)
(``sfr``, fem/fem_e002.c:53-66); the brick goes (-1,-1,-1),(1,-1,-1),
(1,1,-1),(-1,1,-1) and the same four at z=+1 (``e009_fill_coords``,
fem/fem_e009.c:36-70).

Load types: 1 = prescribed displacement (support), 3 = nodal force
(``femApplyNBC``/``femApplyNLoad``, fem/fem_loads.c:343-470).  Directions:
1=UX, 2=UY, 3=UZ (fem/fem_elem.h:44-46).
"""
from __future__ import annotations

import dataclasses
import numpy as np

ELEM_QUAD = 2      # 4-node plane quad, fem/fem_e002.c
ELEM_BRICK = 9     # 8-node brick, fem/fem_e009.c
ELEM_BRICK_W = 10  # brick + Winkler foundation, fem/fem_e010.c
MAT_ISO = 1        # linear isotropic material, fem/fem_m001.c
MAT_STRENGTH = 5   # isotropic with strengths (DENS, EX, NU, G, F_YC, F_YT, F_UC, F_UT), fem/fem_m005.c

# Monte Carlo variable types, fem/fem_mont.h:28-47
MONTE_VTYPE_RS = 0
MONTE_VTYPE_MAT = 1
MONTE_VTYPE_N = 2
MONTE_VTYPE_NLD = 3
MONTE_VTYPE_RES_D = 8
MONTE_VTYPE_RES_R = 9
MONTE_VTYPE_RES_E = 10
MONTE_VTYPE_MAX_D = 7
MONTE_VTYPE_RES_SUM_E = 11
MONTE_VTYPE_RES_MAX_E = 12
MONTE_VTYPE_RES_MIN_E = 13
MONTE_VTYPE_RES_FAIL_E = 14
MONTE_VTYPE_RES_D_MAX = 15
MONTE_VTYPE_RES_D_MIN = 16
MONTE_VTYPE_RES_D_SUM = 17
MONTE_VTYPE_RES_A_MAX = 18
MONTE_VTYPE_RES_FAIL = 19

MAT_EX = 2     # fem/fem_mat.h:41
MAT_F_YC = 12  # fem/fem_mat.h:51
# element result codes, fem/fem_eres.h:39-51
RES_SX, RES_SY, RES_SZ, RES_SXY, RES_SYZ, RES_SZX = 7, 8, 9, 10, 11, 12
RES_EX, RES_EY, RES_EZ, RES_EXY, RES_EYZ, RES_EZX = 13, 14, 15, 16, 17, 18
RES_S1 = 19


@dataclasses.dataclass
class Model:
    n_xyz: np.ndarray            # (nLen, 3) float64
    e_type: np.ndarray           # (eLen,) int64
    e_rs: np.ndarray             # (eLen,) int64, real set position
    e_mp: np.ndarray             # (eLen,) int64, material position
    e_nodes: np.ndarray          # (eLen, nodes_per_elem) int64 node positions
    rs_type: np.ndarray          # (rsLen,) int64
    rs_vals: list                # list of 1-D float arrays
    mp_type: np.ndarray          # (mpLen,) int64
    mp_vals: list                # list of 1-D float arrays (DENS, EX, NU, ...)
    nl_node: np.ndarray          # (nlLen,) int64
    nl_type: np.ndarray
    nl_dir: np.ndarray
    nl_val: np.ndarray           # float64
    mc_vars: np.ndarray | None = None   # (ilen+olen, 5) int64 MC variable table
    mc_ilen: int = 0
    mc_olen: int = 0
    name: str = ""

    # -- flat views in the reference's layout ---------------------------------
    @property
    def nLen(self) -> int:
        return int(self.n_xyz.shape[0])

    @property
    def eLen(self) -> int:
        return int(self.e_type.shape[0])

    def e_from(self) -> np.ndarray:
        cnt = np.full(self.eLen, self.e_nodes.shape[1], dtype=np.int64)
        return np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.int64)

    def rs_flat(self):
        cnt = np.array([len(v) for v in self.rs_vals], dtype=np.int64)
        frm = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.int64)
        vals = np.concatenate([np.asarray(v, np.float64) for v in self.rs_vals]) if cnt.sum() else np.zeros(0)
        return frm, cnt, vals

    def mp_flat(self):
        cnt = np.array([len(v) for v in self.mp_vals], dtype=np.int64)
        frm = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.int64)
        vals = np.concatenate([np.asarray(v, np.float64) for v in self.mp_vals])
        return frm, cnt, vals

    @property
    def dofs_per_node(self) -> int:
        return 2 if int(self.e_type[0]) == ELEM_QUAD else 3

    def n_active_dofs(self) -> int:
        used = np.zeros(self.nLen, dtype=bool)
        used[self.e_nodes.ravel()] = True
        return int(used.sum()) * self.dofs_per_node


def _fmt(x: float) -> str:
    return repr(float(x))


def write_fem(model: Model, path: str) -> None:
    """Write ``model`` as a preparsed uFEM input file (fem/feminput.5).

    Section order follows ``femReadInput`` (fem/fem_io.c:380-590) and the
    readers it calls: solution control, real sets, materials, nodes, elements,
    gravity, nodal loads, element loads (``femReadInputLoads``, :86), the
    three transient counters (``femReadRepeatData``, :167), the dynamics count
    (``femReadInputDynLoads``, :297) and, when present, the Monte Carlo
    variable table (``fem_monte_read_data``, fem/fem_mont.c:866).
    """
    out = []
    w = out.append
    w("1 -1\n1 0 1\n")
    rs_frm, rs_cnt, rs_vals = model.rs_flat()
    w(f"{len(model.rs_type)}\n")
    for i, t in enumerate(model.rs_type):
        w(f"{i + 1} {int(t)} {int(rs_cnt[i])}\n")
    w(f"{int(rs_cnt.sum())}\n")
    if len(rs_vals):
        w("\n".join(_fmt(v) for v in rs_vals) + "\n")
    mp_frm, mp_cnt, mp_vals = model.mp_flat()
    w(f"{len(model.mp_type)}\n")
    w("".join(f"{i + 1} {int(t)} {int(mp_cnt[i])}\n" for i, t in enumerate(model.mp_type)))
    w(f"{int(mp_cnt.sum())}\n")
    w("\n".join(_fmt(v) for v in mp_vals) + "\n")
    w(f"{model.nLen}\n")
    xyz = model.n_xyz
    w("".join(f"{i + 1} {_fmt(xyz[i, 0])} {_fmt(xyz[i, 1])} {_fmt(xyz[i, 2])}\n" for i in range(model.nLen)))
    w(f"{model.eLen}\n")
    nn = model.e_nodes.shape[1]
    w("".join(f"{i + 1} {int(model.e_type[i])} {int(model.e_rs[i])} {int(model.e_mp[i])} {nn}\n"
              for i in range(model.eLen)))
    w(f"{model.eLen * nn}\n")
    w("\n".join(" ".join(str(int(v)) for v in row) for row in model.e_nodes) + "\n")
    w("0 0.0\n")
    w(f"{len(model.nl_node)}\n")
    w("".join(f"{int(model.nl_node[i])} {int(model.nl_type[i])} {int(model.nl_dir[i])} {_fmt(model.nl_val[i])}\n"
              for i in range(len(model.nl_node))))
    w("0\n0 0 0\n0\n")
    if model.mc_vars is not None and model.mc_ilen > 0:
        w(f"{model.mc_ilen} {model.mc_olen}\n")
        w("".join(" ".join(str(int(v)) for v in row) + "\n" for row in model.mc_vars))
    with open(path, "w") as f:
        f.write("".join(out))


# ----------------------------------------------------------------------------
# generators
# ----------------------------------------------------------------------------

def plate_quad(nx=64, ny=16, lx=4.0, ly=1.0, thick=0.2, E=30e9, nu=0.2, total_load=-100e3,
               distort=0.0, seed=0) -> Model:
    """2-D cantilever plate of 4-node quads.

    Left edge (x=0) fixed in UX and UY; ``total_load`` in UY split equally over
    the right-edge nodes.  ``distort`` moves interior nodes by a seeded random
    fraction of the element size, for parity tests on non-rectangular
    elements.
    """
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    xyz = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    if distort:
        rng = np.random.default_rng(seed)
        ix = np.tile(np.arange(nx + 1), ny + 1)
        iy = np.repeat(np.arange(ny + 1), nx + 1)
        inner = (ix > 0) & (ix < nx) & (iy > 0) & (iy < ny)
        d = rng.uniform(-distort, distort, size=(xyz.shape[0], 2)) * np.array([lx / nx, ly / ny])
        xyz[inner, :2] += d[inner]
    nid = lambda i, j: j * (nx + 1) + i
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    I = I.ravel(); J = J.ravel()
    en = np.stack([nid(I, J), nid(I + 1, J), nid(I + 1, J + 1), nid(I, J + 1)], axis=1).astype(np.int64)
    ne = en.shape[0]
    left = np.array([nid(0, j) for j in range(ny + 1)])
    right = np.array([nid(nx, j) for j in range(ny + 1)])
    nl_node = np.concatenate([np.repeat(left, 2), right])
    nl_type = np.concatenate([np.ones(2 * len(left)), np.full(len(right), 3)]).astype(np.int64)
    nl_dir = np.concatenate([np.tile([1, 2], len(left)), np.full(len(right), 2)]).astype(np.int64)
    nl_val = np.concatenate([np.zeros(2 * len(left)), np.full(len(right), total_load / len(right))])
    return Model(
        n_xyz=xyz, e_type=np.full(ne, ELEM_QUAD, np.int64), e_rs=np.zeros(ne, np.int64),
        e_mp=np.zeros(ne, np.int64), e_nodes=en,
        rs_type=np.array([ELEM_QUAD], np.int64), rs_vals=[np.array([thick])],
        mp_type=np.array([MAT_ISO], np.int64), mp_vals=[np.array([2500.0, E, nu])],
        nl_node=nl_node.astype(np.int64), nl_type=nl_type, nl_dir=nl_dir, nl_val=nl_val,
        name=f"plate_{nx}x{ny}")


def _brick_grid(nx, ny, nz, lx, ly, lz, distort=0.0, seed=0):
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    if distort:
        rng = np.random.default_rng(seed)
        iz, iy, ix = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
        inner = ((ix > 0) & (ix < nx) & (iy > 0) & (iy < ny) & (iz > 0) & (iz < nz)).ravel()
        d = rng.uniform(-distort, distort, size=xyz.shape) * np.array([lx / nx, ly / ny, lz / nz])
        xyz[inner] += d[inner]
    nid = lambda i, j, k: (k * (ny + 1) + j) * (nx + 1) + i
    K_, J_, I_ = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    I_ = I_.ravel(); J_ = J_.ravel(); K_ = K_.ravel()
    en = np.stack([nid(I_, J_, K_), nid(I_ + 1, J_, K_), nid(I_ + 1, J_ + 1, K_), nid(I_, J_ + 1, K_),
                   nid(I_, J_, K_ + 1), nid(I_ + 1, J_, K_ + 1), nid(I_ + 1, J_ + 1, K_ + 1),
                   nid(I_, J_ + 1, K_ + 1)], axis=1).astype(np.int64)
    return xyz, en, nid


def _lumped_face(n1, n2, h1, h2, mask1=None, mask2=None):
    """Bilinear lumping weights (corner 1/4, edge 1/2, interior 1) x h1*h2."""
    w1 = np.ones(n1 + 1); w1[0] = w1[-1] = 0.5
    w2 = np.ones(n2 + 1); w2[0] = w2[-1] = 0.5
    if mask1 is not None:
        w1 = mask1
    if mask2 is not None:
        w2 = mask2
    return np.outer(w2, w1) * h1 * h2   # [i2, i1]


def beam_brick(nx=80, ny=20, nz=20, lx=8.0, ly=2.0, lz=2.0, E=30e9, nu=0.2, traction=1e6,
               per_element_material=False, zones=0, distort=0.0, seed=0) -> Model:
    """3-D cantilever beam of 8-node bricks.

    The x=0 face is fixed in UX, UY, UZ (type-1 supports, value 0).  A uniform
    traction ``traction`` [Pa] acts in -z on the x=lx face, lumped to its nodes
    with bilinear weights.  ``per_element_material`` gives every element its
    own material record (the reference randomises material values per
    material, fem/fem_mont.c:721-736, so per-element E needs one record per
    element); ``zones`` > 0 instead gives ``zones`` equal-length materials
    along x.
    """
    xyz, en, nid = _brick_grid(nx, ny, nz, lx, ly, lz, distort, seed)
    ne = en.shape[0]
    fixed = np.array([nid(0, j, k) for k in range(nz + 1) for j in range(ny + 1)])
    hy, hz = ly / ny, lz / nz
    w = _lumped_face(ny, nz, hy, hz)          # [k, j]
    tip = np.array([[nid(nx, j, k) for j in range(ny + 1)] for k in range(nz + 1)])
    nl_node = np.concatenate([np.repeat(fixed, 3), tip.ravel()])
    nl_type = np.concatenate([np.ones(3 * len(fixed)), np.full(tip.size, 3)]).astype(np.int64)
    nl_dir = np.concatenate([np.tile([1, 2, 3], len(fixed)), np.full(tip.size, 3)]).astype(np.int64)
    nl_val = np.concatenate([np.zeros(3 * len(fixed)), -traction * w.ravel()])
    if per_element_material:
        e_mp = np.arange(ne, dtype=np.int64)
        mp_vals = [np.array([2500.0, E, nu]) for _ in range(ne)]
    elif zones:
        ix = np.arange(ne) % nx
        e_mp = (ix * zones // nx).astype(np.int64)
        mp_vals = [np.array([2500.0, E, nu]) for _ in range(zones)]
    else:
        e_mp = np.zeros(ne, np.int64)
        mp_vals = [np.array([2500.0, E, nu])]
    return Model(
        n_xyz=xyz, e_type=np.full(ne, ELEM_BRICK, np.int64), e_rs=np.zeros(ne, np.int64),
        e_mp=e_mp, e_nodes=en,
        rs_type=np.array([ELEM_BRICK], np.int64), rs_vals=[np.zeros(0)],
        mp_type=np.full(len(mp_vals), MAT_ISO, np.int64), mp_vals=mp_vals,
        nl_node=nl_node.astype(np.int64), nl_type=nl_type, nl_dir=nl_dir, nl_val=nl_val,
        name=f"beam_{nx}x{ny}x{nz}")


def block_brick(nx=128, ny=128, nz=64, lx=12.8, ly=12.8, lz=6.4, E=30e9, nu=0.25, pressure=0.5e6,
                patch=3.2) -> Model:
    """3-D block on a fixed base (z=0 face fixed) with a centred square
    pressure patch of side ``patch`` on the top face, lumped bilinearly."""
    xyz, en, nid = _brick_grid(nx, ny, nz, lx, ly, lz)
    ne = en.shape[0]
    fixed = np.array([nid(i, j, 0) for j in range(ny + 1) for i in range(nx + 1)])
    hx, hy = lx / nx, ly / ny
    lo_x, hi_x = (lx - patch) / 2, (lx + patch) / 2
    lo_y, hi_y = (ly - patch) / 2, (ly + patch) / 2
    ix0, ix1 = int(round(lo_x / hx)), int(round(hi_x / hx))
    iy0, iy1 = int(round(lo_y / hy)), int(round(hi_y / hy))
    wx = np.zeros(nx + 1); wx[ix0:ix1 + 1] = 1.0; wx[ix0] = wx[ix1] = 0.5
    wy = np.zeros(ny + 1); wy[iy0:iy1 + 1] = 1.0; wy[iy0] = wy[iy1] = 0.5
    w = np.outer(wy, wx) * hx * hy
    js, is_ = np.nonzero(w)
    top = np.array([nid(i, j, nz) for j, i in zip(js, is_)])
    nl_node = np.concatenate([np.repeat(fixed, 3), top])
    nl_type = np.concatenate([np.ones(3 * len(fixed)), np.full(len(top), 3)]).astype(np.int64)
    nl_dir = np.concatenate([np.tile([1, 2, 3], len(fixed)), np.full(len(top), 3)]).astype(np.int64)
    nl_val = np.concatenate([np.zeros(3 * len(fixed)), -pressure * w[js, is_]])
    return Model(
        n_xyz=xyz, e_type=np.full(ne, ELEM_BRICK, np.int64), e_rs=np.zeros(ne, np.int64),
        e_mp=np.zeros(ne, np.int64), e_nodes=en,
        rs_type=np.array([ELEM_BRICK], np.int64), rs_vals=[np.zeros(0)],
        mp_type=np.array([MAT_ISO], np.int64), mp_vals=[np.array([2500.0, E, nu])],
        nl_node=nl_node.astype(np.int64), nl_type=nl_type, nl_dir=nl_dir, nl_val=nl_val,
        name=f"block_{nx}x{ny}x{nz}")


# ----------------------------------------------------------------------------
# Monte Carlo sampling
# ----------------------------------------------------------------------------

MC_SEED = 20261203


def mc_rng(mesh_id: int, sample: int, seed: int = MC_SEED) -> np.random.Generator:
    """One counter-based Philox stream per (mesh, sample), keyed by ``seed``."""
    key = np.array([seed, (mesh_id << 32) | sample], dtype=np.uint64)
    return np.random.Generator(np.random.Philox(key=key))


def mc_attach_vars(model: Model, kind: str = "element_E", n_out_nodes: int = 4) -> Model:
    """Attach a Monte Carlo variable table to ``model`` (fem/fem_mont.c:866).

    Inputs: E of every material (``MONTE_VTYPE_MAT``, subitem MAT_EX) and the
    value of every type-3 nodal force (``MONTE_VTYPE_NLD``).  Outputs: UZ at
    ``n_out_nodes`` tip nodes (``MONTE_VTYPE_RES_D``) and the UX/UZ
    reactions of the first support node (``MONTE_VTYPE_RES_R``).
    """
    rows = []
    for m in range(len(model.mp_vals)):
        rows.append([len(rows), MONTE_VTYPE_MAT, m, MAT_EX, 0])
    force_idx = np.nonzero(model.nl_type == 3)[0]
    for i in force_idx:
        rows.append([len(rows), MONTE_VTYPE_NLD, int(model.nl_node[i]), 3, int(model.nl_dir[i])])
    ilen = len(rows)
    tip_nodes = model.nl_node[force_idx]
    pick = tip_nodes[np.linspace(0, len(tip_nodes) - 1, n_out_nodes).astype(int)]
    out = []
    for n in pick:
        out.append([len(out), MONTE_VTYPE_RES_D, int(n), 3, 0])
    sup = int(model.nl_node[np.nonzero(model.nl_type == 1)[0][0]])
    out.append([len(out), MONTE_VTYPE_RES_R, sup, 1, 0])
    out.append([len(out), MONTE_VTYPE_RES_R, sup, 3, 0])
    model.mc_vars = np.array(rows + out, dtype=np.int64)
    model.mc_ilen = ilen
    model.mc_olen = len(out)
    return model


def mc_attach_outputs(model: Model) -> Model:
    """Attach a Monte Carlo table that asks for every linear-static output of
    ``monte_fill_ofld_data`` (fem/fem_mont.c:514-686) and the general failure
    function (fem/fem_asse.c:271-374).

    Inputs: E of every material, F_YC of every material record that holds one
    (type 5), every type-3 nodal force, and MAX_D.  Outputs (written to
    permuted positions): RES_D, RES_R, D_MAX/D_MIN/D_SUM/A_MAX at the last
    loaded node; RES_E at stored and unstored result points (point 0, the
    last stored point and the one after it, a result code the element never
    writes); SUM/MAX/MIN/FAIL_E over stress, strain and unwritten codes; and
    RES_FAIL.
    """
    quad = int(model.e_type[0]) == ELEM_QUAD
    rows = []
    for m in range(len(model.mp_vals)):
        rows.append([MONTE_VTYPE_MAT, m, MAT_EX, 0])
        if int(model.mp_type[m]) == MAT_STRENGTH and len(model.mp_vals[m]) > 4:
            rows.append([MONTE_VTYPE_MAT, m, MAT_F_YC, 0])
    force_idx = np.nonzero(model.nl_type == 3)[0]
    for i in force_idx:
        rows.append([MONTE_VTYPE_NLD, int(model.nl_node[i]), 3, int(model.nl_dir[i])])
    rows.append([MONTE_VTYPE_MAX_D, 0, 0, 0])
    ilen = len(rows)
    tip, tdir = int(model.nl_node[force_idx[-1]]), int(model.nl_dir[force_idx[-1]])
    sup = int(model.nl_node[np.nonzero(model.nl_type == 1)[0][0]])
    ne = model.eLen
    last = ne - 1
    # result points the element stores (fem/fem_e002.c:942, fem/fem_e009.c:825, fem/fem_e010.c:41)
    npt = 4 if quad else (22 if int(model.e_type[last]) == ELEM_BRICK_W else 19)
    npt0 = 4 if quad else (22 if int(model.e_type[0]) == ELEM_BRICK_W else 19)
    out = [[MONTE_VTYPE_RES_D, tip, tdir, 0], [MONTE_VTYPE_RES_R, sup, 1, 0],
           [MONTE_VTYPE_RES_D_MAX, tip, tdir, 0], [MONTE_VTYPE_RES_D_MIN, tip, tdir, 0],
           [MONTE_VTYPE_RES_D_SUM, tip, tdir, 0], [MONTE_VTYPE_RES_A_MAX, tip, tdir, 0],
           [MONTE_VTYPE_RES_E, 0, RES_SX, 1], [MONTE_VTYPE_RES_E, 0, RES_SXY, npt0],
           [MONTE_VTYPE_RES_E, last, RES_EX, 2], [MONTE_VTYPE_RES_E, last, RES_EXY, 3],
           [MONTE_VTYPE_RES_E, 0, RES_SX, 0], [MONTE_VTYPE_RES_E, last, RES_SY, npt],
           [MONTE_VTYPE_RES_E, last, RES_SY, npt + 1], [MONTE_VTYPE_RES_E, ne // 2, RES_S1, 1]]
    codes = [RES_SX, RES_SXY, RES_EX, RES_EY, RES_S1]
    if not quad:
        out += [[MONTE_VTYPE_RES_E, 0, RES_SZ, npt0], [MONTE_VTYPE_RES_E, last, RES_EYZ, 7],
                [MONTE_VTYPE_RES_E, last, RES_EZX, npt], [MONTE_VTYPE_RES_E, 0, RES_SZX, 27]]
        codes += [RES_SZ, RES_SYZ, RES_EZX]
    for c in codes:
        for t in (MONTE_VTYPE_RES_SUM_E, MONTE_VTYPE_RES_MAX_E, MONTE_VTYPE_RES_MIN_E, MONTE_VTYPE_RES_FAIL_E):
            out.append([t, 0, c, 0])
    out.append([MONTE_VTYPE_RES_FAIL, 0, 0, 0])
    olen = len(out)
    table = [[i] + r for i, r in enumerate(rows)] + [[olen - 1 - j] + r for j, r in enumerate(out)]
    model.mc_vars = np.array(table, dtype=np.int64)
    model.mc_ilen = ilen
    model.mc_olen = olen
    return model


def mc_outputs_samples(model: Model, nsamp: int, vm_scale: float, u_scale: float,
                       mesh_id: int = 77, E0: float = 30e9, sigma: float = 0.15) -> np.ndarray:
    """Seeded inputs for ``mc_attach_outputs``' table: E lognormal around E0,
    one load factor U(0.8, 1.2) for every force, F_YC = vm_scale x r1 (one
    r1 per sample for every material) and MAX_D = u_scale x r2, each r drawn
    from U(0.5, 0.9) or U(1.15, 2) (so that about half of the samples fail
    each test)."""
    ty = model.mc_vars[:model.mc_ilen, 1]
    sub = model.mc_vars[:model.mc_ilen, 3]
    is_force = ty == MONTE_VTYPE_NLD
    nl = {(int(n), int(d)): float(v) for n, t, d, v in
          zip(model.nl_node, model.nl_type, model.nl_dir, model.nl_val) if t == 3}
    ifld = np.empty((nsamp, model.mc_ilen), dtype=np.float64)
    for s in range(nsamp):
        g = mc_rng(mesh_id, s)
        lf = g.uniform(0.8, 1.2)
        r1, r2 = (g.uniform(0.5, 0.9) if g.uniform() < 0.5 else g.uniform(1.15, 2.0) for _ in range(2))
        for i in range(model.mc_ilen):
            if ty[i] == MONTE_VTYPE_MAT and sub[i] == MAT_EX:
                ifld[s, i] = E0 * np.exp(sigma * g.standard_normal())
            elif ty[i] == MONTE_VTYPE_MAT:
                ifld[s, i] = vm_scale * r1 * g.uniform(0.95, 1.05)
            elif is_force[i]:
                ifld[s, i] = nl[(int(model.mc_vars[i, 2]), int(model.mc_vars[i, 4]))] * lf
            else:
                ifld[s, i] = u_scale * r2
    return ifld


def mc_samples(model: Model, mesh_id: int, nsamp: int, first_sample: int = 0,
               E0: float = 30e9, sigma: float = 0.15, mean_one: bool = True,
               load_lo: float = 0.8, load_hi: float = 1.2) -> np.ndarray:
    """Seeded input rows ``ifld[nsamp, ilen]`` for ``model``'s MC table.

    Each material gets E = E0 * exp(sigma*z - sigma^2/2) (``mean_one``) or
    E0 * exp(sigma*z) (median E0), z iid N(0,1); every nodal force is the
    model's base value times one load factor ~ U(load_lo, load_hi) per sample.
    """
    nmat = len(model.mp_vals)
    force_idx = np.nonzero(model.nl_type == 3)[0]
    base = model.nl_val[force_idx]
    shift = -0.5 * sigma * sigma if mean_one else 0.0
    ifld = np.empty((nsamp, nmat + len(force_idx)), dtype=np.float64)
    for s in range(nsamp):
        g = mc_rng(mesh_id, first_sample + s)
        z = g.standard_normal(nmat)
        lf = g.uniform(load_lo, load_hi)
        ifld[s, :nmat] = E0 * np.exp(sigma * z + shift)
        ifld[s, nmat:] = base * lf
    return ifld


def warm_beam(nx=40, ny=10, nz=10, zones=16, lx=8.0, ly=2.0, lz=2.0, n_out_nodes=4) -> Model:
    """The learned-warm-start beam: ``zones`` equal-length materials along x,
    with the Monte Carlo table of ``mc_attach_vars`` (E of every zone, then the
    value of every tip force)."""
    m = beam_brick(nx, ny, nz, lx, ly, lz, zones=zones)
    return mc_attach_vars(m, n_out_nodes=n_out_nodes)


def warm_features(model: Model):
    """Network inputs of the warm start: the zone E values as compliances 1/E
    (displacements of an elastic body are close to linear in them: for a
    statically determinate beam, exactly so in beam theory) and the first tip
    force (all tip forces share one random load factor) as log|.|, and the
    solution's scale column (the first tip force: u is linear in it)."""
    nmat = len(model.mp_vals)
    cols = list(range(nmat)) + [nmat]
    return cols, [2] * nmat + [1], nmat


def warm_samples(model: Model, nsamp: int, first_sample: int = 0, mesh_id: int = 5) -> np.ndarray:
    """Warm-start inputs: zone E = 30 GPa * exp(0.15 z) (median 30 GPa), load
    factor U(0.8, 1.2).  Training and evaluation draw disjoint sample ids."""
    return mc_samples(model, mesh_id=mesh_id, nsamp=nsamp, first_sample=first_sample, mean_one=False)


def model_for_sample(model: Model, row) -> Model:
    """A copy of ``model`` with one Monte Carlo sample's inputs applied, as
    monte_solution applies ifld before solving (fem/fem_mont.c:715-800): E
    of materials (``MONTE_VTYPE_MAT`` / MAT_EX) and nodal force values
    (``MONTE_VTYPE_NLD``)."""
    import copy
    ms = copy.deepcopy(model)
    ms.mp_vals = [v.copy() for v in model.mp_vals]
    ms.nl_val = model.nl_val.copy()
    for var in model.mc_vars[:model.mc_ilen]:
        pos, ty, item, sub, it = [int(x) for x in var]
        if ty == MONTE_VTYPE_MAT and sub == MAT_EX:
            ms.mp_vals[item][1] = row[pos]
        elif ty == MONTE_VTYPE_NLD:
            for j in range(len(ms.nl_node)):
                if ms.nl_node[j] == item and ms.nl_type[j] == sub and ms.nl_dir[j] == it:
                    ms.nl_val[j] = row[pos]
                    break
    return ms
