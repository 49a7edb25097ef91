"""The Monte Carlo output pass (fem/fem_mont.c:514-686) and the failure
function (fem/fem_asse.c): the oracle's restatement against the reference
library's own outputs, then (GPU) the per-sample and batched plugin paths
against the same fixtures."""
import math

import numpy as np
import pytest

from golden_util import load, model_from

CASES = ["mc_out_plate_6x3", "mc_out_beam_4x2x2", "mc_out_plate_iso_4x2"]


def _fail_col(z):
    il, ol = int(z["mc_ilen"]), int(z["mc_olen"])
    j = [j for j in range(ol) if int(z["mc_vars"][il + j][1]) == 19][0]
    return int(z["mc_vars"][j][0])


@pytest.mark.parametrize("name", CASES)
def test_restatement_matches_reference(name):
    """Every output of every sample, bit for bit (the oracle solves with the
    reference's SSOR PCG and iteration cap, so u is the reference's)."""
    from oracle.mc_outputs import monte_run
    z = load(name)
    out = monte_run(model_from(z), z["ifld"])
    assert np.array_equal(out, z["ofld"])


def test_fixtures_exercise_each_failure_test():
    """Across the fixtures some samples pass RES_FAIL, some fail only the
    strength test, some only the displacement test (sqrt(max|u|) >= MAX_D)."""
    from oracle import mc_outputs as mo
    from oracle.oracle import EPS_REF, SOLVER_SSOR, OracleModel
    kinds = set()
    for name in CASES[:2]:
        z = load(name)
        m0 = model_from(z)
        for s in range(z["ifld"].shape[0]):
            m, md = mo.apply_inputs(m0, z["ifld"][s])
            om = OracleModel(m)
            om.dofs(); om.fill_K(); om.loads_bcs()
            om.solve(SOLVER_SSOR, EPS_REF, max_it=3 * om.rows)
            u = om.get_u()
            sig, _, _ = om.results()
            fy = [mo.mat_value(m.mp_type[m.e_mp[e]], m.mp_vals[m.e_mp[e]], mo.MAT_F_YC) for e in range(m.eLen)]
            strength = mo.fail_cond(m.e_type, fy, sig, om.strains())
            disp = int(math.sqrt(np.abs(u).max()) >= md)
            kinds.add((strength, disp))
            assert z["ofld"][s, _fail_col(z)] == float(strength or disp)
    assert {(0, 0), (1, 0), (0, 1)} <= kinds


def test_type1_material_always_fails():
    """A type-1 record holds no F_YC, so femGetMPValPos gives 0 and the von
    Mises test fails at result set 0 (fem/fem_asse.c:59-75)."""
    z = load("mc_out_plate_iso_4x2")
    assert np.all(z["ofld"][:, _fail_col(z)] == 1.0)


# ---- GPU: the plugin paths against the reference library's outputs ---------

def _columns(z):
    """Per output j: (ofld column, type, code) -- the column comes from row j of
    the table, as the reference reads it (fem/fem_mont.c:522 and on)."""
    il, ol = int(z["mc_ilen"]), int(z["mc_olen"])
    mv = z["mc_vars"]
    return [(int(mv[j][0]), int(mv[il + j][1]), int(mv[il + j][3])) for j in range(ol)]


def _stored_total(m):
    return int(sum({2: 4, 9: 19, 10: 22}[int(t)] for t in m.e_type))


def _compare(out, ref, z, rtol, cumulative_reactions):
    """out/ref: [nsamp, olen].  Flags and D_SUM exactly; sums within rtol of
    max(|MAX|, |MIN|) x stored points of the same code; reactions per sample
    (the reference accumulates them: consecutive differences); the rest within
    rtol of the column's largest magnitude (0 where the reference gives 0)."""
    cols = _columns(z)
    n = _stored_total(model_from(z))
    by_code = {}
    for c, t, code in cols:
        by_code[(t, code)] = c
    ref = np.array(ref, np.float64)
    for c, t, code in cols:
        r, o = ref[:, c].copy(), out[:, c]
        if t == 9 and cumulative_reactions:
            r = np.diff(np.concatenate([[0.0], r]))
        if t in (14, 17, 19):
            assert np.array_equal(o, r), (c, t, code, o, r)
        elif t == 11:
            bound = np.maximum(np.abs(ref[:, by_code[(12, code)]]), np.abs(ref[:, by_code[(13, code)]])) * n
            assert np.all(np.abs(o - r) <= rtol * bound + 1e-300), (c, code, o, r)
        else:
            scale = np.abs(r).max()
            assert np.all(np.abs(o - r) <= rtol * scale), (c, t, code, o, r)


@pytest.fixture(scope="module")
def fem_paths(tmp_path_factory):
    from ufem_b200 import meshgen as mg
    d = tmp_path_factory.mktemp("mcout")
    out = {}
    for name in CASES:
        z = load(name)
        p = str(d / f"{name}.fem")
        mg.write_fem(model_from(z), p)
        out[name] = (z, p)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_plugin_outputs_match_reference(fem_paths, name):
    """monte_solution, one sample per call: every output type against the
    reference library, the failure flags exactly."""
    from ufem_b200.mc import MonteLib
    z, path = fem_paths[name]
    lib = MonteLib(path)
    try:
        assert lib.ffunc == int(z["ffunc"])
        out = np.zeros_like(z["ofld"])
        for s in range(z["ifld"].shape[0]):
            rv, out[s] = lib.solution(z["ifld"][s])
            assert rv == 0
        _compare(out, z["ofld"], z, 1e-8, cumulative_reactions=True)
    finally:
        lib.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_batch_outputs_match_reference(fem_paths, name):
    """monte_solution_batch: the fused element pass over all samples at once
    (F_YC and MAX_D as per-sample input columns)."""
    from ufem_b200.mc import MonteLib
    z, path = fem_paths[name]
    lib = MonteLib(path)
    try:
        rv, out, st = lib.solution_batch(z["ifld"])
        assert rv == 0 and (st == 0).all()
        _compare(out, z["ofld"], z, 1e-6, cumulative_reactions=True)
        rv, out2, _ = lib.solution_batch(z["ifld"])
        assert np.array_equal(out, out2)  # run-to-run identical
    finally:
        lib.close()


@pytest.mark.gpu
def test_serial_outputs_match_reference(fem_paths):
    """ufem_mc_solve_serial (the per-sample loop behind the plain bench arm)."""
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve_serial
    z, _ = fem_paths["mc_out_beam_4x2x2"]
    g = GpuModel(model_from(z))
    out, st, _ = mc_solve_serial(g, z["ifld"], tol=1e-10)
    assert (st == 0).all()
    _compare(out, z["ofld"], z, 1e-6, cumulative_reactions=True)


@pytest.mark.gpu
def test_batch_failure_many_samples(fem_paths):
    """256 samples (two sample groups of 128) through the batched pass against
    per-sample monte_solution calls: every output, flags exactly."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.mc import MonteLib
    z, path = fem_paths["mc_out_beam_4x2x2"]
    m = model_from(z)
    ifld = mg.mc_outputs_samples(m, 256, vm_scale=float(np.median(z["ifld"][:, 1])),
                                 u_scale=float(np.median(z["ifld"][:, -1])), mesh_id=91)
    lib = MonteLib(path)
    try:
        rv, ob, st = lib.solution_batch(ifld)
        assert rv == 0 and (st == 0).all()
        single = np.zeros_like(ob)
        for s in range(ifld.shape[0]):
            rv, single[s] = lib.solution(ifld[s])
        cols = _columns(z)
        fail_col = [c for c, t, _ in cols if t == 19][0]
        assert 0 < single[:, fail_col].sum() < ifld.shape[0]
        _compare(ob, single, z, 1e-6, cumulative_reactions=False)
    finally:
        lib.close()
