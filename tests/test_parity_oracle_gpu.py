"""Parity of the batched, warm-started Monte Carlo path with the FP64 oracle
at 1e-8, and of the 80x20x20 beam (config 2) with the reference's solver.

The warm-start workload's beam (40x10x10 bricks, 16 lognormal E zones and a
load factor, 14,883 DOFs) is trained once (POD basis, MLP, coarse space of
the preconditioner); 256 fresh samples are solved by

  A. the POD-Galerkin guess + FP64 implicit batched PCG with the coarse
     correction,
  B. the MLP guess + FP32 PCG with FP64 solution and true-residual
     replacement (precision 1), and
  C. the MLP guess + FP32 implicit batched PCG (FP32 work vectors, blocks
     formed in the kernel in FP64, FP64 solution and true-residual
     replacement) with the coarse correction (precision 3), and the same
     with FP32 SpMV products (precision 4, the bench headline's form),

each with the stopping rule tightened to a true relative residual of 1e-10
(the FP64 floor of |f - K u| / |f| on this beam is about 1e-11:
|K| |u| / |f| is 1.9e6).
Eight samples spread over the 128-sample groups are solved by the oracle
(oracle/ufem_oracle.c: the reference's assembly and femEqsCGwJ with its own
stopping rule, fem/fem_eqs.c:88-247).  Checked against it:

  * displacements: max |u - u_oracle| / max |u_oracle| <= 1e-8, for the full
    u of the warm-started batched solve (guess from ufem_warm_guess, then
    ufem_mc_solve_device from it) and for the tip outputs of ufem_warm_solve;
  * von Mises stress at the brick's stored result points (1-19,
    fem/fem_e009.c:825), from the GPU result pass on the batched u against
    the oracle's from its own u: max |vm - vm_oracle| / max |vm_oracle| <= 1e-8.
"""
import copy

import numpy as np
import pytest

from golden_util import load, model_sha

pytestmark = pytest.mark.gpu

TOL = 1e-8          # the north_star's displacement and stress bar
SOLVE_TOL = 1e-10   # true relative residual of the GPU solves checked here
PICK = (0, 37, 101, 128, 170, 200, 233, 255)


def _model_for_sample(m, row):
    """The model with one sample's inputs applied (zone E, forces)."""
    from ufem_b200 import meshgen as mg
    ms = copy.deepcopy(m)
    ms.mp_vals = [v.copy() for v in m.mp_vals]
    ms.nl_val = m.nl_val.copy()
    for var in m.mc_vars[:m.mc_ilen]:
        pos, ty, item, sub, it = [int(x) for x in var]
        if ty == mg.MONTE_VTYPE_MAT and sub == mg.MAT_EX:
            ms.mp_vals[item][1] = row[pos]
        elif ty == mg.MONTE_VTYPE_NLD:
            for j in range(len(ms.nl_node)):
                if ms.nl_node[j] == item and ms.nl_type[j] == sub and ms.nl_dir[j] == it:
                    ms.nl_val[j] = row[pos]
                    break
    return ms


def _von_mises(sig):
    """von Mises stress of (SX, SY, SZ, SYZ, SZX, SXY) records."""
    sx, sy, sz, syz, szx, sxy = (sig[..., k] for k in range(6))
    return np.sqrt(0.5 * ((sx - sy) ** 2 + (sy - sz) ** 2 + (sz - sx) ** 2) + 3.0 * (sxy ** 2 + syz ** 2 + szx ** 2))


@pytest.fixture(scope="module")
def warm40():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.warm import WarmStart
    from oracle.oracle import OracleModel
    m = mg.warm_beam(40, 10, 10, zones=16)
    g = GpuModel(m)
    cols, logs, sc = mg.warm_features(m)
    ws = WarmStart(g, cols, logs, sc, n_modes=64, n_hidden=128, n_snapshots=512, epochs=60, batch=256, lr=2e-3,
                   n_coarse=64)
    st = ws.train(mg.warm_samples(m, 1024), precision=2)
    ev = mg.warm_samples(m, 256, first_sample=1 << 20)
    oracle = {}
    for s in PICK:
        ms = _model_for_sample(m, ev[s])
        o = OracleModel(ms).run_static()
        assert o["rv_solve"] == 0
        oracle[s] = (ms, o["u"], _von_mises(o["sig"][:, :19, :]), o["ndoffld"])
    return m, g, ws, st, ev, oracle


def _solve_from(g, ifld, u0, precision, tol):
    """ufem_mc_solve_device from the guesses u0 [nsamp][ndof]: (u [nsamp][ndof], status, iters)."""
    import ctypes as C
    import torch
    from ufem_b200 import _lib
    from ufem_b200.mc import default_options
    L = _lib.load()
    n = ifld.shape[0]
    S = max(128, (n + 127) // 128 * 128)
    d_in = torch.from_numpy(np.ascontiguousarray(ifld)).cuda()
    d_out = torch.zeros((n, max(1, g.model.mc_olen)), dtype=torch.float64, device="cuda")
    d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_it = torch.zeros(n, dtype=torch.int64, device="cuda")
    g0 = np.zeros((g.ndof, S))
    g0[:, :n] = u0.T  # the device guess layout: [nDOFAct][S], sample fastest
    d_g = torch.from_numpy(g0).cuda()
    d_u = torch.zeros((g.ndof, S), dtype=torch.float64, device="cuda")
    vp = lambda t: (C.c_void_p * 1)(t.data_ptr())
    opt = default_options()
    opt.precision = precision
    opt.tol = tol
    opt.coarse = 1
    rv = L.ufem_mc_solve_device(1, (C.c_void_p * 1)(g.h.value), np.array([n], np.int64).ctypes.data_as(
        C.POINTER(C.c_long)), vp(d_in), vp(d_out), vp(d_st), vp(d_it), vp(d_g), vp(d_u), C.byref(opt))
    _lib.check("ufem_mc_solve_device", rv)
    return d_u[:, :n].T.cpu().numpy(), d_st.cpu().numpy(), d_it.cpu().numpy()


def _gpu_von_mises(ms, u):
    """von Mises at the stored points from the GPU result pass on u."""
    from ufem_b200.api import GpuModel
    gs = GpuModel(ms)
    gs.fill_K(0)
    gs.add_loads()
    gs.add_disps()
    gs.set_u(u)
    gs.fill_K(1)
    _, vm = gs.stresses(ms.eLen, False)
    return np.asarray(vm).reshape(ms.eLen, 27)[:, :19]


def _check_against_oracle(m, ev, u, oracle, label):
    worst_u = worst_vm = 0.0
    for s in PICK:
        ms, uo, vmo, _ = oracle[s]
        eu = float(np.abs(u[s] - uo).max() / np.abs(uo).max())
        vm = _gpu_von_mises(ms, u[s])
        evm = float(np.abs(vm - vmo).max() / np.abs(vmo).max())
        worst_u, worst_vm = max(worst_u, eu), max(worst_vm, evm)
    assert worst_u <= TOL, (label, worst_u)
    assert worst_vm <= TOL, (label, worst_vm)
    return worst_u, worst_vm


def _check_outputs(m, ev, of, oracle, label):
    """RES_D outputs (tip UZ) of the warm solve against the oracle's u."""
    from ufem_b200 import meshgen as mg
    rows = [(j, int(r[2]), int(r[3])) for j, r in enumerate(m.mc_vars[m.mc_ilen:]) if r[1] == mg.MONTE_VTYPE_RES_D]
    worst = 0.0
    for s in PICK:
        _, uo, _, nd = oracle[s]
        pos = [int(m.mc_vars[m.mc_ilen + j][0]) for j, _, _ in rows]
        want = np.array([uo[nd[node * 7 + d - 1] - 1] for _, node, d in rows])
        got = of[s, pos]
        worst = max(worst, float(np.abs(got - want).max() / np.abs(want).max()))
    assert worst <= TOL, (label, worst)


def test_galerkin_fp64_coarse_within_1e8_of_oracle(warm40):
    m, g, ws, st, ev, oracle = warm40
    assert st["coarse_modes"] >= 16
    ws.set_guess_mode(1)
    try:
        u0 = ws.guess(ev)
        u, status, iters = _solve_from(g, ev, u0, precision=2, tol=SOLVE_TOL)
        of, st_w, it_w, wst = ws.solve(ev, precision=2, tol=SOLVE_TOL)
    finally:
        ws.set_guess_mode(0)
    assert (status == 0).all()
    assert np.isin(st_w, [0, 4]).all()
    _check_against_oracle(m, ev, u, oracle, "Galerkin + FP64 implicit + coarse")
    _check_outputs(m, ev, of, oracle, "Galerkin + FP64 implicit + coarse, ufem_warm_solve")


def test_mlp_fp32_fp64_within_1e8_of_oracle(warm40):
    m, g, ws, st, ev, oracle = warm40
    ws.set_guess_mode(0)
    u0 = ws.guess(ev)
    u, status, iters = _solve_from(g, ev, u0, precision=1, tol=SOLVE_TOL)
    of, st_w, it_w, wst = ws.solve(ev, precision=1, tol=SOLVE_TOL)
    assert (status == 0).all()
    assert np.isin(st_w, [0, 4]).all()
    _check_against_oracle(m, ev, u, oracle, "MLP + FP32/FP64")
    _check_outputs(m, ev, of, oracle, "MLP + FP32/FP64, ufem_warm_solve")


def test_mlp_fp32_implicit_coarse_within_1e8_of_oracle(warm40):
    m, g, ws, st, ev, oracle = warm40
    ws.set_guess_mode(0)
    u0 = ws.guess(ev)
    u, status, iters = _solve_from(g, ev, u0, precision=3, tol=SOLVE_TOL)
    of, st_w, it_w, wst = ws.solve(ev, precision=3, tol=SOLVE_TOL)
    assert (status == 0).all()
    assert np.isin(st_w, [0, 4]).all()
    _check_against_oracle(m, ev, u, oracle, "MLP + FP32 implicit + coarse")
    _check_outputs(m, ev, of, oracle, "MLP + FP32 implicit + coarse, ufem_warm_solve")


def test_mlp_fp32_products_coarse_within_1e8_of_oracle(warm40):
    """Precision 4: FP32 SpMV products (the inner FP32 matrix) with the warm
    start and the coarse correction, FP64 true-residual replacement."""
    m, g, ws, st, ev, oracle = warm40
    ws.set_guess_mode(0)
    u0 = ws.guess(ev)
    u, status, iters = _solve_from(g, ev, u0, precision=4, tol=SOLVE_TOL)
    of, st_w, it_w, wst = ws.solve(ev, precision=4, tol=SOLVE_TOL)
    assert (status == 0).all()
    assert np.isin(st_w, [0, 4]).all()
    _check_against_oracle(m, ev, u, oracle, "MLP + FP32 products + coarse")
    _check_outputs(m, ev, of, oracle, "MLP + FP32 products + coarse, ufem_warm_solve")


def test_beam_80x20x20_within_1e8_of_reference():
    """Config 2 (107,163 DOFs): the FP64 PCG with the reference's stopping
    rule, and the FP64 PCG to a relative residual of 1e-10, against the
    reference's own displacements (tests/golden/beam_80x20x20.npz, made by
    make_golden.py with the reference's femEqsCGwJ)."""
    import hashlib
    from ufem_b200 import api, meshgen as mg
    from ufem_b200.api import GpuModel
    z = load("beam_80x20x20")
    m = mg.beam_brick(80, 20, 20, 8.0, 2.0, 2.0)
    assert model_sha(m) == str(z["model_sha"])
    u_ref = z["u"]
    g = GpuModel(m)
    nd = g.ndoffld(m.nLen)
    assert hashlib.sha256(np.ascontiguousarray(nd, np.int64).tobytes()).hexdigest() == str(z["ndoffld_sha"])
    rv, it = g.fem_solve()
    assert rv == 0
    e_ref = float(np.abs(g.u() - u_ref).max() / np.abs(u_ref).max())
    assert e_ref <= TOL, e_ref
    g.set_u(np.zeros(g.ndof))
    g.solve(api.SOLVER_CGWJ, api.STOP_RELRES, SOLVE_TOL, 0)
    e_tight = float(np.abs(g.u() - u_ref).max() / np.abs(u_ref).max())
    assert e_tight <= TOL, e_tight
