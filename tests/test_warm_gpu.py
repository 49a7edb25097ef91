"""Learned warm start on the GPU (no counterpart in the reference).

* the FP64 GEMM and the one-block Jacobi eigen kernel against numpy;
* the POD basis against numpy's SVD of the same snapshots: orthonormal to
  1e-10, snapshot projection error within 1 % of the optimal rank-r error
  (or below 1e-18 of the snapshots' energy, their own solve accuracy);
* the warm-started batched solve against cold batched solves of the same
  samples: outputs within 1e-6 relative (both stop at true relative
  residual 1e-8; the tip displacements amplify that by the conditioning, as
  in the other Monte Carlo tests), fewer iterations on average, guess error
  reported;
* the fallback: guesses made bad on purpose (scaled by 1e6) regress past the
  cold iteration cap, every sample is solved again from zero and reported
  UFEM_ST_FALLBACK, with the same outputs.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ST_CONVERGED, ST_FALLBACK = 0, 4


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("M,N,K", [(300, 70, 5000), (64, 64, 16), (1000, 130, 100), (17, 5, 3000)])
def test_dgemm_f64_matches_numpy(M, N, K):
    import torch
    from ufem_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(M * 7 + N)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    dC = torch.zeros((M, N), dtype=torch.float64, device="cuda")
    _lib.check("ufem_dgemm_f64", L.ufem_dgemm_f64(M, N, K, dA.data_ptr(), dB.data_ptr(), dC.data_ptr()))
    ref = A @ B
    scale = np.abs(A) @ np.abs(B)
    assert (np.abs(dC.cpu().numpy() - ref) / scale).max() < 1e-13


@pytest.mark.parametrize("l", [8, 80, 96, 98, 144])
def test_sym_eig_matches_numpy(l):
    from ufem_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(l)
    Qm, _ = np.linalg.qr(rng.standard_normal((l, l)))
    lam = np.concatenate([np.geomspace(1e6, 1e-6, l - 4), [3.0, 3.0, 0.0, -2.0]])  # repeated and zero
    A = (Qm * lam) @ Qm.T
    A = 0.5 * (A + A.T)
    V = np.zeros((l, l))
    w = np.zeros(l)
    sw = C.c_int()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    _lib.check("ufem_sym_eig", L.ufem_sym_eig(l, dp(np.ascontiguousarray(A)), dp(V), dp(w), C.byref(sw)))
    nA = np.abs(lam).max()
    assert np.abs(A @ V - V * w).max() <= 1e-12 * nA
    assert np.abs(V.T @ V - np.eye(l)).max() <= 1e-12
    assert np.abs(np.sort(w) - np.sort(np.linalg.eigvalsh(A))).max() <= 1e-12 * nA
    assert sw.value < 60


@pytest.fixture(scope="module")
def warm_small():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.warm import WarmStart
    m = mg.warm_beam(12, 3, 3, zones=4)
    g = GpuModel(m)
    cols, logs, scale_col = mg.warm_features(m)
    ws = WarmStart(g, cols, logs, scale_col, n_modes=32, n_snapshots=256, epochs=150, batch=128, lr=2e-3)
    train = mg.warm_samples(m, 768)
    stats = ws.train(train)
    return m, g, ws, train, stats


def _cold_solutions(g, ifld):
    """Cold batched FP32/FP64 solves through ufem_mc_solve_device: u [nsamp][ndof]."""
    import torch
    from ufem_b200 import _lib
    from ufem_b200.mc import default_options
    L = _lib.load()
    n = ifld.shape[0]
    S = max(128, (n + 127) // 128 * 128)
    d_in = torch.from_numpy(np.ascontiguousarray(ifld)).cuda()
    d_out = torch.zeros((n, g.model.mc_olen), dtype=torch.float64, device="cuda")
    d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_it = torch.zeros(n, dtype=torch.int64, device="cuda")
    d_u = torch.zeros((g.ndof, S), dtype=torch.float64, device="cuda")
    vp = lambda t: (C.c_void_p * 1)(t.data_ptr())
    opt = default_options()
    rv = L.ufem_mc_solve_device(1, (C.c_void_p * 1)(g.h.value), np.array([n], np.int64).ctypes.data_as(
        C.POINTER(C.c_long)), vp(d_in), vp(d_out), vp(d_st), vp(d_it), (C.c_void_p * 1)(), vp(d_u), C.byref(opt))
    _lib.check("ufem_mc_solve_device", rv)
    assert (d_st.cpu().numpy() == ST_CONVERGED).all()
    return d_u[:, :n].T.cpu().numpy(), d_out.cpu().numpy(), d_it.cpu().numpy()


def test_training_reduces_loss(warm_small):
    m, g, ws, train, st = warm_small
    assert st["loss_last"] < 0.1 * st["loss_first"]
    assert st["cold_iters_max"] > 0


def test_basis_orthonormal_and_near_optimal(warm_small):
    m, g, ws, train, st = warm_small
    phi, s2 = ws.basis()
    r = phi.shape[1]
    # modes beyond the snapshots' numerical rank (1e-12 of the largest
    # singular value) are zero columns; the others are orthonormal
    live = np.abs(phi).max(axis=0) > 0
    assert live[:4].all() and (np.diff(live.astype(int)) <= 0).all()
    gram = phi.T @ phi
    assert np.abs(gram - np.diag(live.astype(float))).max() < 1e-10
    U, _, _ = _cold_solutions(g, train[:256])
    U = U.T  # [ndof][nsnap]
    sv = np.linalg.svd(U, compute_uv=False)
    opt_err = np.sum(sv[r:] ** 2)
    got_err = np.sum((U - phi @ (phi.T @ U)) ** 2)
    # within 1 % of the optimal rank-r error, or below the snapshots' own
    # accuracy (they solve to relative residual 1e-8: energy floor 1e-18)
    assert got_err <= 1.01 * opt_err + 1e-18 * np.sum(sv ** 2)
    big = sv[:r] > 1e-4 * sv[0]
    assert np.abs(s2[:r][big] - sv[:r][big] ** 2).max() <= 1e-6 * sv[0] ** 2
    assert (~live <= (sv[:r] < 1e-10 * sv[0])).all()  # only negligible modes may be missing


def test_warm_solve_matches_cold_and_saves_iterations(warm_small):
    from ufem_b200 import meshgen as mg
    m, g, ws, train, st = warm_small
    ev = mg.warm_samples(m, 256, first_sample=1 << 20)
    of, status, iters, wst = ws.solve(ev)
    _, of_cold, it_cold = _cold_solutions(g, ev)
    assert np.isin(status, [ST_CONVERGED, ST_FALLBACK]).all()
    assert _rel(of, of_cold) < 1e-6
    assert iters.mean() < it_cold.mean()
    assert wst["guess_err_mean"] < 0.05
    assert wst["fallbacks"] == int((status == ST_FALLBACK).sum())


def test_fallback_on_bad_guesses(warm_small):
    from ufem_b200 import meshgen as mg
    m, g, ws, train, st = warm_small
    ev = mg.warm_samples(m, 64, first_sample=1 << 21)
    ws.set_guess_scale(1e6)
    try:
        of, status, iters, wst = ws.solve(ev)
    finally:
        ws.set_guess_scale(1.0)
    _, of_cold, _ = _cold_solutions(g, ev)
    assert (status == ST_FALLBACK).all()
    assert wst["fallbacks"] == 64
    assert _rel(of, of_cold) < 1e-6


def test_guess_deterministic(warm_small):
    from ufem_b200 import meshgen as mg
    m, g, ws, train, st = warm_small
    ev = mg.warm_samples(m, 40, first_sample=1 << 22)
    a = ws.guess(ev)
    b = ws.guess(ev)
    assert np.array_equal(a, b)
    assert a.shape == (40, g.ndof)


def test_network_improves_on_its_least_squares_part(warm_small):
    """The guess is a least-squares quadratic model of the POD coefficients
    plus the trained network's correction: with the network (guess mode 0)
    the mean guess error is below that of the least-squares part alone
    (mode 2), and the outputs agree with cold solves."""
    from ufem_b200 import meshgen as mg
    m, g, ws, train, st = warm_small
    ev = mg.warm_samples(m, 256, first_sample=1 << 25)
    ws.set_guess_mode(2)
    try:
        of_l, st_l, it_l, ws_l = ws.solve(ev)
    finally:
        ws.set_guess_mode(0)
    of_m, st_m, it_m, ws_m = ws.solve(ev)
    _, of_cold, it_cold = _cold_solutions(g, ev)
    assert ws_m["guess_err_mean"] < ws_l["guess_err_mean"]
    assert ws_m["guess_err_mean"] < 1e-4
    assert np.isin(st_m, [ST_CONVERGED, ST_FALLBACK]).all() and np.isin(st_l, [ST_CONVERGED, ST_FALLBACK]).all()
    assert _rel(of_m, of_cold) < 1e-6 and _rel(of_l, of_cold) < 1e-6
    assert it_m.mean() < it_cold.mean()


def test_galerkin_guess_beats_the_mlp(warm_small):
    """Guess mode 1 (each sample's POD-Galerkin coefficients from the
    per-variable reduced operators Phi^T K_v Phi): a far smaller guess error
    than the MLP's, fewer PCG iterations, the same outputs as a cold solve."""
    from ufem_b200 import meshgen as mg
    m, g, ws, train, st = warm_small
    ev = mg.warm_samples(m, 128, first_sample=1 << 23)
    of_m, st_m, it_m, ws_m = ws.solve(ev)
    ws.set_guess_mode(1)
    try:
        of_g, st_g, it_g, ws_g = ws.solve(ev)
    finally:
        ws.set_guess_mode(0)
    _, of_cold, it_cold = _cold_solutions(g, ev)
    assert np.isin(st_g, [ST_CONVERGED, ST_FALLBACK]).all()
    assert ws_g["guess_err_mean"] < 1e-2 * ws_m["guess_err_mean"]
    assert it_g.mean() < it_m.mean() < it_cold.mean()
    assert _rel(of_g, of_cold) < 1e-6


def test_galerkin_guess_equals_dense_projection(warm_small):
    """The reduced system built from the per-variable operators equals the
    Galerkin projection with the sample's assembled stiffness: the guess is
    Phi (Phi^T K Phi)^-1 Phi^T f, checked in numpy on the GPU's own K."""
    import scipy.sparse.linalg as spl
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from test_mc_gpu import model_from_sample
    m, g, ws, train, st = warm_small
    ev = mg.warm_samples(m, 3, first_sample=1 << 24)
    ws.set_guess_mode(1)
    try:
        u0 = ws.guess(ev)
    finally:
        ws.set_guess_mode(0)
    phi, _ = ws.basis()
    for s in range(3):
        gs = GpuModel(model_from_sample(m, ev[s]))
        gs.fill_K(0)
        gs.add_loads()
        gs.add_disps()
        b, nbr, nnzb = gs.bsr_shape()
        rp, ci = gs.bsr_pattern()
        vals = gs.K_values()
        from scipy.sparse import csr_matrix
        rows = np.repeat(np.arange(nbr), np.diff(rp))
        r_idx = (rows[:, None, None] * b + np.arange(b)[None, :, None]) + 0 * np.arange(b)[None, None, :]
        c_idx = (ci[:, None, None] * b + np.arange(b)[None, None, :]) + 0 * np.arange(b)[None, :, None]
        K = csr_matrix((vals.ravel(), (r_idx.ravel(), c_idx.ravel())), shape=(gs.ndof, gs.ndof))
        live = np.abs(phi).max(axis=0) > 0
        P = phi[:, live]
        c = np.linalg.solve(P.T @ (K @ P), P.T @ gs.F())
        ref = P @ c
        assert np.abs(u0[s] - ref).max() <= 1e-8 * np.abs(ref).max()
