"""GPU parity of the static path against the reference (golden fixtures) and
the bit-exact oracle restatement.

Bars (the north-star's): DOF numbering and sparsity pattern bit-exact;
element matrices within 1e-12 relative (max-norm over the element); K within
1e-12 relative; displacements within 1e-8 relative of the reference's own
solver; stresses and reactions within 1e-8 relative (they follow u).
"""
import numpy as np
import pytest

from golden_util import STATIC_CASES, load, model_from
from oracle.oracle import OracleModel

pytestmark = pytest.mark.gpu

KE_TOL = 1e-12
K_TOL = 1e-12
U_TOL = 1e-8


def gpu_model(model):
    from ufem_b200.api import GpuModel
    return GpuModel(model)


def relerr(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", STATIC_CASES)
def test_dofs_and_pattern_bitexact(name):
    z = load(name)
    model = model_from(z)
    g = gpu_model(model)
    assert g.ndof == len(z["u"])
    assert np.array_equal(g.ndoffld(model.nLen), z["ndoffld"])
    fp, dp, pos = g.rowslot()
    assert np.array_equal(fp, z["K_frompos"])
    assert np.array_equal(dp, z["K_defpos"])
    assert np.array_equal(pos, z["K_pos"])
    # the GPU block pattern holds exactly the reference's (row, col) set
    b, nbr, nnzb = g.bsr_shape()
    rp, ci = g.bsr_pattern()
    ref_pairs = set()
    for i in range(len(fp)):
        for j in range(fp[i], fp[i] + dp[i]):
            if pos[j] <= 0:
                break
            ref_pairs.add((i, pos[j] - 1))
    gpu_pairs = set()
    for I in range(nbr):
        for k in range(rp[I], rp[I + 1]):
            for a in range(b):
                for c in range(b):
                    gpu_pairs.add((I * b + a, ci[k] * b + c))
    assert gpu_pairs == ref_pairs


@pytest.mark.parametrize("name", STATIC_CASES)
def test_element_matrices(name):
    z = load(name)
    model = model_from(z)
    g = gpu_model(model)
    sz = 8 if int(model.e_type[0]) == 2 else 24
    ke = g.element_matrices(model.eLen, sz)
    ref = z["Ke"]
    idx = z["Ke_idx"] if "Ke_idx" in z.files else np.arange(model.eLen)
    for j, e in enumerate(idx):
        assert relerr(ke[e], ref[j]) <= KE_TOL, (name, e, relerr(ke[e], ref[j]))
    # every element against the oracle restatement (bit-exact with the reference)
    om = OracleModel(model)
    om.dofs()
    worst = max(relerr(ke[e], om.elem_ke(e)) for e in range(model.eLen))
    assert worst <= KE_TOL, worst
    # exact symmetry of the GPU element matrices
    assert np.array_equal(ke, np.transpose(ke, (0, 2, 1)))


@pytest.mark.parametrize("name", ["plate_6x3_distorted", "plate_4x2_strain", "brick_3x2x2_distorted",
                                  "plate_4x2_prescribed"])
def test_assembly_and_supports(name):
    from ufem_b200.api import bsr_to_dense, rowslot_to_dense
    z = load(name)
    model = model_from(z)
    g = gpu_model(model)
    b, nbr, nnzb = g.bsr_shape()
    rp, ci = g.bsr_pattern()
    g.fill_K(0)
    K = bsr_to_dense(rp, ci, g.K_values(), b)
    Kref = rowslot_to_dense(z["K_frompos"], z["K_defpos"], z["K_pos"], z["K_data"])
    assert relerr(K, Kref) <= K_TOL
    assert np.array_equal(K, K.T)                 # deterministic symmetric assembly
    g.add_loads()
    assert np.array_equal(g.F(), z["F_loads"])    # host sums in the reference's order
    g.add_disps()
    Kbc = bsr_to_dense(rp, ci, g.K_values(), b)
    Kbc_ref = rowslot_to_dense(z["K_frompos"], z["K_defpos"], z["K_pos"], z["Kbc_data"])
    assert relerr(Kbc, Kbc_ref) <= K_TOL
    assert relerr(g.F(), z["F_bc"]) <= K_TOL


@pytest.mark.parametrize("name", STATIC_CASES)
def test_fem_solve_matches_reference(name):
    z = load(name)
    model = model_from(z)
    g = gpu_model(model)
    rv, it = g.fem_solve(check=False)
    u = g.u()
    uref = z["u"]
    if int(z["rv_solve"]) == 0:
        assert rv == 0, (name, rv, it)
        assert relerr(u, uref) <= U_TOL, (name, relerr(u, uref))
    else:
        # the reference stops with AF_ERR at maxIt = nDOFAct on this tiny model
        # (its 1e-21 test sits at round-off); the iterate still agrees closely.
        # femSolve skips the result pass then, so run it here for the check.
        assert relerr(u, uref) <= 1e-6
        g.fill_K(1)
    quad = int(model.e_type[0]) == 2
    sig, vm = g.stresses(model.eLen, quad)
    nst = 4 if quad else 19
    ref = z["eres"][:, :nst]
    assert relerr(sig[:, :nst], ref) <= (U_TOL if int(z["rv_solve"]) == 0 else 1e-6)
    # von Mises from the stresses (invariant form of fdb/fdb_cres.c:404-435)
    if quad:
        sx, sy, t = sig[..., 0], sig[..., 1], sig[..., 2]
        vm_ref = np.sqrt(sx * sx - sx * sy + sy * sy + 3 * t * t)
    else:
        sx, sy, sz, tyz, tzx, txy = [sig[..., k] for k in range(6)]
        vm_ref = np.sqrt(0.5 * ((sx - sy) ** 2 + (sy - sz) ** 2 + (sz - sx) ** 2) + 3 * (tyz ** 2 + tzx ** 2 + txy ** 2))
    assert relerr(vm, vm_ref) <= 1e-12
    node, dof, val = g.reactions()
    assert np.array_equal(node, z["reac_node"]) and np.array_equal(dof, z["reac_dof"])
    assert relerr(val, z["reac_val"]) <= (U_TOL if int(z["rv_solve"]) == 0 else 1e-6)


def test_stresses_all_points_vs_oracle():
    """All 27 brick points (the reference stores 19) against the oracle."""
    z = load("brick_3x2x2_distorted")
    model = model_from(z)
    g = gpu_model(model)
    g.fem_solve()
    om = OracleModel(model)
    o = om.run_static()
    sig, _ = g.stresses(model.eLen, False)
    assert relerr(sig, o["sig"]) <= U_TOL


@pytest.mark.parametrize("name", ["plate_6x3_distorted", "brick_3x2x2_distorted"])
@pytest.mark.parametrize("solver", ["ssor", "bicg"])
def test_solver_variants(name, solver):
    from ufem_b200 import api
    z = load(name)
    model = model_from(z)
    g = gpu_model(model)
    g.fill_K(0)
    g.add_loads()
    g.add_disps()
    code = api.SOLVER_SSOR if solver == "ssor" else api.SOLVER_BICG
    rv, it = g.solve(code, api.STOP_RELRES, 1e-12, 10 * g.ndof, check=False)
    assert rv == 0
    assert relerr(g.u(), z[f"u_{solver}"]) <= U_TOL


@pytest.mark.parametrize("which", ["cgwj", "bicg", "ssor"])
def test_level1_dropin_on_rowslot_matrix(which):
    """femEqs* replacements on the reference's own tMatrix arrays."""
    from ufem_b200 import api
    z = load("brick_3x2x2_distorted")
    eps = api.EPS_REF if which == "cgwj" else 1e-14
    rv, x = api.eqs(which, z["K_frompos"], z["K_defpos"], z["K_pos"], z["Kbc_data"], z["F_bc"],
                    np.zeros(len(z["F_bc"])), eps=eps, max_it=20 * len(z["F_bc"]))
    assert rv == 0
    assert relerr(x, z["u"]) <= U_TOL


def test_dropin_error_codes():
    from ufem_b200 import api
    z = load("plate_4x2_strain")
    fp, dp, pos = z["K_frompos"], z["K_defpos"], z["K_pos"]
    data = z["Kbc_data"].copy()
    for j in range(fp[5], fp[5] + dp[5]):
        if pos[j] == 6:
            data[j] = 0.0
    rv, _ = api.eqs("cgwj", fp, dp, pos, data, z["F_bc"], np.zeros(len(fp)))
    assert rv == -13                                 # AF_ERR_ZER
    rv, x = api.eqs("cgwj", fp, dp, pos, z["Kbc_data"], np.zeros(len(fp)), np.ones(len(fp)))
    assert rv == 0 and not x.any()                   # zero load: x = 0
    rv, _ = api.eqs("cgwj", fp, dp, pos, z["Kbc_data"], z["F_bc"], np.zeros(len(fp)), max_it=1)
    assert rv == -1                                  # AF_ERR, unconverged


def test_inverted_element_is_rejected():
    from ufem_b200 import meshgen as mg
    from ufem_b200._lib import UfemError
    m = mg.beam_brick(2, 1, 1, 1.0, 0.5, 0.5)
    m.e_nodes = m.e_nodes.copy()
    m.e_nodes[0] = m.e_nodes[0][[4, 5, 6, 7, 0, 1, 2, 3]]   # upside down: detJ < 0
    g = gpu_model(m)
    with pytest.raises(UfemError) as ei:
        g.fill_K(0)
    assert ei.value.rv == -3                         # AF_ERR_VAL (fem/fem_e009.c:87-94)


def test_run_twice_bitwise_identical():
    from ufem_b200 import meshgen as mg
    m = mg.beam_brick(10, 3, 3, 4.0, 1.0, 1.0, distort=0.2, seed=2)
    outs = []
    for _ in range(2):
        g = gpu_model(m)
        g.fem_solve()
        outs.append((g.K_values().copy(), g.u()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_beam_80x20x20_true_residual():
    """Config 2 (107,163 DOFs): FP64 PCG to relative residual 1e-10, checked
    by a size-independent property: |f - K u| / |f| from the GPU K in numpy."""
    from scipy.sparse import csr_matrix
    from ufem_b200 import api, meshgen as mg
    m = mg.beam_brick(80, 20, 20, 8.0, 2.0, 2.0)
    g = gpu_model(m)
    assert g.ndof == 107163
    g.fill_K(0)
    g.add_loads()
    g.add_disps()
    rv, it = g.solve(api.SOLVER_CGWJ, api.STOP_RELRES, 1e-10, 0)
    assert rv == 0
    b, nbr, nnzb = g.bsr_shape()
    rp, ci = g.bsr_pattern()
    vals = g.K_values()
    rows = np.repeat(np.arange(nbr), np.diff(rp))
    r_idx = (rows[:, None, None] * 3 + np.arange(3)[None, :, None]) + 0 * np.arange(3)[None, None, :]
    c_idx = (ci[:, None, None] * 3 + np.arange(3)[None, None, :]) + 0 * np.arange(3)[None, :, None]
    K = csr_matrix((vals.ravel(), (r_idx.ravel(), c_idx.ravel())), shape=(g.ndof, g.ndof))
    f = g.F()
    u = g.u()
    assert np.linalg.norm(f - K @ u) / np.linalg.norm(f) <= 1e-10
    # cantilever sanity: tip deflection is downward and of the beam-theory size
    assert u.min() < 0


def _assembled_csr(g):
    from scipy.sparse import csr_matrix
    b, nbr, nnzb = g.bsr_shape()
    rp, ci = g.bsr_pattern()
    vals = g.K_values()
    rows = np.repeat(np.arange(nbr), np.diff(rp))
    r_idx = (rows[:, None, None] * b + np.arange(b)[None, :, None]) + 0 * np.arange(b)[None, None, :]
    c_idx = (ci[:, None, None] * b + np.arange(b)[None, None, :]) + 0 * np.arange(b)[None, :, None]
    return csr_matrix((vals.ravel(), (r_idx.ravel(), c_idx.ravel())), shape=(g.ndof, g.ndof))


@pytest.mark.parametrize("shape", [(20, 5, 5), (80, 20, 20)])
def test_mixed_precision_pcg(shape):
    """PCG on the FP32 matrix copy with FP64 true-residual replacement
    (UFEM_SOLVER_CGWJ_MIXED) to true relative residual 1e-8, checked in numpy
    with the GPU's FP64 K, and against the plain FP64 PCG solution to 1e-10
    (displacements within 1e-6 relative)."""
    from ufem_b200 import api, meshgen as mg
    m = mg.beam_brick(*shape, 8.0, 2.0, 2.0)
    ref = gpu_model(m)
    ref.fill_K(0)
    ref.add_loads()
    ref.add_disps()
    ref.solve(api.SOLVER_CGWJ, api.STOP_RELRES, 1e-10, 0)
    u64 = ref.u()
    g = gpu_model(m)
    g.fill_K(0)
    g.add_loads()
    g.add_disps()
    rv, it = g.solve(api.SOLVER_CGWJ_MIXED, api.STOP_RELRES, 1e-8, 0)
    assert rv == 0 and it > 0
    K = _assembled_csr(g)
    f, u = g.F(), g.u()
    assert np.linalg.norm(f - K @ u) / np.linalg.norm(f) <= 1e-8
    assert np.abs(u - u64).max() <= 1e-6 * np.abs(u64).max()
