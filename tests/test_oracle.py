"""The oracle restatement against the reference's own outputs.

The fixtures in tests/golden/ were produced by the unmodified reference
(oracle/_ref built from its sources, tests/golden/make_golden.py).  The
restatement reproduces every intermediate bit for bit: element matrices, the
DOF map, the row-slot pattern in first-touch order, K before and after the
supports, the load vector, the CG/SSOR/BiCGStab solutions, reactions and the
stored integration-point stresses.
"""
import hashlib

import numpy as np
import pytest

from golden_util import STATIC_CASES, load, model_from
from oracle.oracle import OracleModel, solve_rowslot


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", STATIC_CASES)
def test_static_bitexact(name):
    z = load(name)
    model = model_from(z)
    om = OracleModel(model)
    o = om.run_static()
    assert np.array_equal(o["ndoffld"], z["ndoffld"])
    for k in ("K_frompos", "K_defpos", "K_pos"):
        assert np.array_equal(o[k], z[k]), k
    assert sha(o["K_data"]) == str(z["sha_K_data"])
    assert sha(o["Kbc_data"]) == str(z["sha_Kbc_data"])
    assert np.array_equal(o["F_loads"], z["F_loads"])
    assert np.array_equal(o["F_bc"], z["F_bc"])
    assert o["rv_solve"] == int(z["rv_solve"])
    assert np.array_equal(o["u"], z["u"])
    assert np.array_equal(o["reac"], z["reac_val"])
    nst = 4 if o["sig"].shape[1] == 4 else 19   # the reference stores brick IPs 1..19 only
    assert np.array_equal(o["sig"][:, :nst], z["eres"][:, :nst])
    if "Ke_idx" in z.files:
        for j, e in enumerate(z["Ke_idx"]):
            assert np.array_equal(om.elem_ke(int(e)), z["Ke"][j])
    else:
        ke = np.stack([om.elem_ke(e) for e in range(model.eLen)])
        assert np.array_equal(ke, z["Ke"])
        assert sha(ke) == str(z["sha_Ke"])


@pytest.mark.parametrize("name", ["plate_6x3_distorted", "brick_3x2x2_distorted"])
@pytest.mark.parametrize("solver", ["ssor", "bicg"])
def test_solver_variants_bitexact(name, solver):
    z = load(name)
    rv, x, _ = solve_rowslot(solver, z["K_frompos"], z["K_defpos"], z["K_pos"], z["Kbc_data"],
                             z["F_bc"], np.zeros(len(z["F_bc"])))
    assert rv == int(z[f"rv_{solver}"])
    assert np.array_equal(x, z[f"u_{solver}"])


def test_unconverged_returns_af_err():
    """maxIt = nDOFAct is too few for 1e-21 on this tiny distorted plate: the
    reference returns AF_ERR (-1, fem/fem_eqs.c:230-236) and so does the oracle."""
    z = load("plate_6x3_distorted")
    assert int(z["rv_solve"]) == -1
    rv, x, it = solve_rowslot("cgwj", z["K_frompos"], z["K_defpos"], z["K_pos"], z["Kbc_data"],
                              z["F_bc"], np.zeros(len(z["F_bc"])))
    assert rv == -1 and it == len(z["F_bc"])


def test_zero_diagonal_af_err_zer():
    """A zero diagonal entry gives AF_ERR_ZER (fem/fem_eqs.c:134-145)."""
    z = load("plate_4x2_strain")
    data = z["Kbc_data"].copy()
    fp, dp, pos = z["K_frompos"], z["K_defpos"], z["K_pos"]
    row = 5
    for j in range(fp[row], fp[row] + dp[row]):
        if pos[j] == row + 1:
            data[j] = 0.0
    rv, _, _ = solve_rowslot("cgwj", fp, dp, pos, data, z["F_bc"], np.zeros(len(z["F_bc"])))
    assert rv == -13


def test_zero_load_returns_zero_solution():
    z = load("plate_4x2_strain")
    rv, x, it = solve_rowslot("cgwj", z["K_frompos"], z["K_defpos"], z["K_pos"], z["Kbc_data"],
                              np.zeros(len(z["F_bc"])), np.ones(len(z["F_bc"])))
    assert rv == 0 and it == 0 and not x.any()


def test_rigid_body_modes_before_supports():
    """K times a rigid translation is zero (to round-off) before supports."""
    z = load("brick_3x2x2_distorted")
    fp, dp, pos, data = z["K_frompos"], z["K_defpos"], z["K_pos"], z["K_data"]
    n = len(fp)
    for d in range(3):
        t = np.zeros(n)
        t[d::3] = 1.0
        y = np.zeros(n)
        for i in range(n):
            for j in range(fp[i], fp[i] + dp[i]):
                if pos[j] <= 0:
                    break
                y[i] += data[j] * t[pos[j] - 1]
        assert np.abs(y).max() < 1e-6 * np.abs(data).max()


def test_patch_constant_strain_brick():
    """A linear displacement field gives the exact constant stress at every IP."""
    from ufem_b200 import meshgen as mg
    m = mg.beam_brick(2, 2, 2, 1.0, 1.0, 1.0, distort=0.2, seed=1)
    om = OracleModel(m)
    om.dofs()
    om.fill_K()
    eps = np.array([1e-4, -2e-4, 3e-4, 0.0, 0.0, 0.0])
    xyz = m.n_xyz
    u = np.zeros((m.nLen, 3))
    u[:, 0] = eps[0] * xyz[:, 0]
    u[:, 1] = eps[1] * xyz[:, 1]
    u[:, 2] = eps[2] * xyz[:, 2]
    import ctypes as C
    from oracle.oracle import lib
    lib().orc_set_u(om.h, np.ascontiguousarray(u.ravel()))
    sig, _, _ = om.results()
    E, nu = 30e9, 0.2
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    expect = lam * eps[:3].sum() + 2 * mu * eps[:3]
    assert np.allclose(sig[:, :, :3], expect, rtol=1e-9)
    assert np.abs(sig[:, :, 3:]).max() < 1e-6 * np.abs(expect).max()


def test_mc_fixture_shapes():
    z = load("mc_beam_4x2x2")
    assert z["ofld"].shape == (4, int(z["mc_olen"]))
    assert (z["rv"] == 0).all()
