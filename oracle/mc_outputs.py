"""Oracle (test infrastructure): the Monte Carlo output pass restated in numpy.

Restates ``monte_fill_ofld_data`` (fem/fem_mont.c:514-686) for the linear
static solution, with the element-result storage rules of the reference and
the general failure function of fem/fem_asse.c.  Tests compare it with the
reference library's own outputs (golden fixtures) and with the GPU path.

Element results (``femGetEResVal``, fem/fem_dama.h:153 -> femGetRepVal,
fem/fem_accs.c:196-277): result set k >= 1 of code c is read at index
idx(c) + res_rp * (k - 1) of the element's record, and reads at or past the
record length (``rvals``) give 0; set 0 asks for a non-repeating value, of
which these elements have none, so it is 0 as well.  The linear result pass
writes only stresses and strains (fem/fem_e002.c:656-673,
fem/fem_e009.c:545-560), so every other code reads 0.
"""
from __future__ import annotations

import math

import numpy as np

KNOWN_DOFS = 7  # fem/fem_elem.h:43

# per element type: (res_rp, rvals, index of each stress/strain code in
# nres_rp) -- fem/fem_e002.c:942,1024-1031; fem/fem_e009.c:825,880-883;
# fem/fem_e010.c:41,82-91
_QUAD_IDX = {7: 0, 8: 1, 10: 2, 13: 3, 14: 4, 16: 5}
_BRICK_IDX = {7: 0, 8: 1, 9: 2, 11: 3, 12: 4, 10: 5, 13: 6, 14: 7, 15: 8, 17: 9, 18: 10, 16: 11}
ELEM_RES = {2: (22, 76, _QUAD_IDX), 9: (20, 14 * 27, _BRICK_IDX), 10: (32, 26 * 27, _BRICK_IDX)}

# component of the stress (codes 7..12) or strain (13..18) vector as the
# oracle lays them out (quad: SX,SY,SXY; brick: SX,SY,SZ,SYZ,SZX,SXY)
_QUAD_COMP = {7: 0, 8: 1, 10: 2, 13: 0, 14: 1, 16: 2}
_BRICK_COMP = {7: 0, 8: 1, 9: 2, 11: 3, 12: 4, 10: 5, 13: 0, 14: 1, 15: 2, 17: 3, 18: 4, 16: 5}

# non-repeating value list of each material type (fem/fem_m001.c:39,
# fem/fem_m004.c:40, fem/fem_m005.c:39)
MAT_VALS = {1: [1, 2, 5, 38, 37, 39, 36],
            4: [1, 2, 5, 6, 18, 19, 12, 20, 30, 31, 36],
            5: [1, 2, 5, 6, 12, 14, 15, 17]}
MAT_F_YC = 12


def mat_value(mp_type: int, vals, code: int) -> float:
    """femGetMPValPos(e, code, 0) (fem/fem_dama.c:410): the value's index in
    the type's non-repeating list; 0 when absent or past the record."""
    lst = MAT_VALS.get(int(mp_type), [])
    if code not in lst:
        return 0.0
    i = lst.index(code)
    return float(vals[i]) if i < len(vals) else 0.0


def elem_value(etype: int, sig_e, eps_e, code: int, k: int) -> float:
    """femGetEResVal(e, code, k) after the linear result pass."""
    if k <= 0:
        return 0.0
    res_rp, rvals, idx = ELEM_RES[int(etype)]
    if code not in idx or idx[code] + res_rp * (k - 1) >= rvals:
        return 0.0
    comp = (_QUAD_COMP if int(etype) == 2 else _BRICK_COMP)[code]
    return float((sig_e if code <= 12 else eps_e)[k - 1, comp])


def _vmis(stress) -> float:
    """sqrt(3 J2) with J2 of stress2D_J2 (fem/fem_ch2d.c:46-57) or
    stress3D_J2 (fem/fem_chen.c:54-74)."""
    if len(stress) == 3:
        sx, sy, txy = stress
        j2 = (((sx - sy) * (sx - sy)) + (sx * sx) + (sy * sy)) / 6.0 + (txy * txy)
    else:
        sx, sy, sz, t4, t5, t6 = stress
        j2 = ((((sx - sy) * (sx - sy)) + ((sy - sz) * (sy - sz)) + ((sz - sx) * (sz - sx))) / 6.0
              + t6 * t6 + t5 * t5 + t4 * t4)
    return math.sqrt(j2 * 3.0) if j2 >= 0.0 else float("nan")


def fail_cond(e_type, e_fy, sig, eps) -> int:
    """fem_asse_fail_cond (fem/fem_asse.c:271-374) for planes and solids: the
    von Mises test of fem_asse_mat_vmis (fem/fem_asse.c:55-75) at result set
    0 and every set 1..res_rp; 1 at the first point with sqrt(3 J2) not below
    |F_YC|."""
    for e in range(len(e_type)):
        t = int(e_type[e])
        codes = [7, 8, 10] if t == 2 else [7, 8, 9, 11, 12, 10]
        fy = abs(e_fy[e])
        res_rp = ELEM_RES[t][0]
        for k in range(0, res_rp + 1):
            st = [elem_value(t, sig[e], eps[e], c, k) for c in codes]
            if not (_vmis(st) < fy):
                return 1
    return 0


def fill_ofld(mc_vars, ilen: int, olen: int, ndoffld, u, e_type, e_fy, sig, eps,
              reac_node, reac_dof, reac_val, max_disp: float, fail_id: int):
    """Outputs of one sample as ``monte_fill_ofld_data`` writes them into a
    zeroed ofld (fem/fem_mont.c:702-705).  ``u`` is the solved vector (1-based
    DOF numbers index it), ``reac_val`` the reactions the reference holds at
    this point (it accumulates them over samples)."""
    ofld = np.zeros(olen)
    ndof_len = len(ndoffld)
    nrows = len(u)
    ne = len(e_type)

    def uget(p):  # femVecGet (fem/fem_math.c:811-819)
        return float(u[p - 1]) if 1 <= p <= nrows else 0.0

    for i in range(ilen, ilen + olen):
        _, ty, item, sub, it = (int(v) for v in mc_vars[i])
        # the reference reads the output position from row i - ilen of the
        # table (monte_io_var_pos[i-monte_i_len], fem/fem_mont.c:522 and on)
        o = int(mc_vars[i - ilen][0])
        if ty == 8:
            pos = item * KNOWN_DOFS + sub - 1
            ofld[o] = 0.0 if pos > ndof_len else uget(int(ndoffld[pos]))
        elif ty in (15, 16, 17):
            pos = item * KNOWN_DOFS + sub - 1
            if pos > ndof_len:
                continue
            pos = int(ndoffld[pos])
            if ty == 15:
                v = uget(pos)
                if ofld[o] < v:
                    ofld[o] = v
            elif ty == 16:
                v = uget(pos)
                if ofld[o] > v:
                    ofld[o] = v
            else:
                ofld[o] += float(ndoffld[pos])
        elif ty == 9:
            for j in range(len(reac_node)):
                if reac_node[j] == item and reac_dof[j] == sub:
                    ofld[o] = reac_val[j]
                    break
        elif ty == 10:
            ofld[o] = elem_value(e_type[item], sig[item], eps[item], sub, it) if 0 <= item < ne else 0.0
        elif ty in (11, 12, 13, 14):
            acc = 0.0
            for e in range(ne):
                t = int(e_type[e])
                for k in range(0, ELEM_RES[t][0] + 1):
                    v = elem_value(t, sig[e], eps[e], sub, k)
                    if ty == 11:
                        acc += v
                    elif ty == 12:
                        acc = v if v > acc else acc
                    elif ty == 13:
                        acc = v if v < acc else acc
                    elif v > 0.0:
                        acc = 1.0
            ofld[o] = acc
        elif ty == 19 and fail_id > -1:
            # fem_asse_max_disp_simple (fem/fem_asse.c:42-47) compares
            # femVecMaxAbs(u), which returns sqrt(max |u_i|) (fem/fem_math.c:2136-2163)
            if max_disp > 0.0 and math.sqrt(float(np.max(np.abs(u)))) >= abs(max_disp):
                ofld[o] = 1.0
            if fail_cond(e_type, e_fy, sig, eps) != 0:
                ofld[o] = 1.0
    return ofld


def apply_inputs(model, row, max_disp: float = 0.0):
    """A copy of ``model`` with one sample's inputs applied as monte_solution
    does (fem/fem_mont.c:707-800): MAT values by the type's value list, the
    first NLD load with node/type/direction, MAX_D.  Returns (model,
    max_disp)."""
    import copy
    m = copy.deepcopy(model)
    m.mp_vals = [np.array(v, np.float64) for v in m.mp_vals]
    m.nl_val = np.array(m.nl_val, np.float64)
    for i in range(model.mc_ilen):
        pos, ty, item, sub, it = (int(v) for v in model.mc_vars[i])
        v = float(row[pos])
        if ty == 1:
            lst = MAT_VALS.get(int(m.mp_type[item]), [])
            if it == 0 and sub in lst and lst.index(sub) < len(m.mp_vals[item]):
                m.mp_vals[item][lst.index(sub)] = v
        elif ty == 3:
            for j in range(len(m.nl_node)):
                if m.nl_node[j] == item and m.nl_type[j] == sub and m.nl_dir[j] == it:
                    m.nl_val[j] = v
                    break
        elif ty == 7:
            max_disp = abs(v)
    return m, max_disp


def monte_run(model, ifld):
    """Every sample of ``ifld`` through the oracle as monte_solution runs it
    (fem/fem_mont.c:694-856): inputs, the linear solve of monte_linear_solver
    (SSOR PCG to FEM_ZERO/10000 with at most 3 x rows iterations, from u = 0,
    fem/fem_mont.c:480-508), the result pass, then the outputs.  Reactions
    accumulate over the samples as the reference's resRval does."""
    from oracle.oracle import EPS_REF, SOLVER_SSOR, OracleModel
    fail_id = -1
    for i in range(model.mc_ilen, model.mc_ilen + model.mc_olen):
        if int(model.mc_vars[i][1]) == 19:
            fail_id = i - model.mc_ilen  # fem/fem_mont.c:903-904
    out = np.zeros((ifld.shape[0], model.mc_olen))
    reac_acc = None
    max_disp = 0.0
    for s in range(ifld.shape[0]):
        m, max_disp = apply_inputs(model, ifld[s], max_disp)
        om = OracleModel(m)
        ndoffld = om.dofs()
        om.fill_K()
        om.loads_bcs()
        om.solve(SOLVER_SSOR, EPS_REF, max_it=3 * om.rows)
        u = om.get_u()
        sig, _, reac = om.results()
        eps = om.strains()
        reac_acc = reac if reac_acc is None else reac_acc + reac
        e_fy = [mat_value(m.mp_type[m.e_mp[e]], m.mp_vals[m.e_mp[e]], MAT_F_YC) for e in range(m.eLen)]
        rn, rd = reaction_slots(m)
        out[s] = fill_ofld(model.mc_vars, model.mc_ilen, model.mc_olen, ndoffld, u, m.e_type, e_fy,
                           sig, eps, rn, rd, reac_acc, max_disp, fail_id)
    return out


def reaction_slots(m):
    """(node, dof) of each reaction slot: one per support load of type 1, 2, 4,
    5, 6 or 7 in load order, except type-1 loads with a nonzero value
    (fem/fem_sol.c:676-720)."""
    t = np.asarray(m.nl_type)
    keep = np.isin(t, [1, 2, 4, 5, 6, 7]) & ~((t == 1) & (np.asarray(m.nl_val) != 0.0))
    return np.asarray(m.nl_node)[keep], np.asarray(m.nl_dir)[keep]
