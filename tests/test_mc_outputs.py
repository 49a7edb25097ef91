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
