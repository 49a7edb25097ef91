"""Coarse correction of the batched PCG's preconditioner (no counterpart in
the reference): M^-1 = D^-1 + Wc Wc^T, both products on the tensor cores.

A preconditioner changes the iterates, not the answer: with a coarse space
every sample still stops at the FP64 true relative residual 1e-8, so
displacements and outputs agree with the Jacobi-only solve within 1e-6
relative (the conditioning allowance of the other Monte Carlo tests).  The
coarse space here is built on the host the way the warm start builds it:
Phi = the leading left singular vectors of FP64 solutions, Wc = Phi L^-T with
L L^T = Phi^T Kbar Phi, Kbar the oracle's stiffness (supports applied) at
the samples' mean inputs.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _solve(g, ifld, coarse=1, precision=2):
    """Batched solve through ufem_mc_solve_device: (u [nsamp][ndof], status,
    iters, ofld, stats)."""
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
    d_u = torch.zeros((g.ndof, S), dtype=torch.float64, device="cuda")
    vp = lambda t: (C.c_void_p * 1)(t.data_ptr())
    opt = default_options()
    opt.precision = precision
    opt.coarse = coarse
    rv = L.ufem_mc_solve_device(1, (C.c_void_p * 1)(g.h.value), np.array([n], np.int64).ctypes.data_as(
        C.POINTER(C.c_long)), vp(d_in), vp(d_out), vp(d_st), vp(d_it), (C.c_void_p * 1)(), vp(d_u), C.byref(opt))
    _lib.check("ufem_mc_solve_device", rv)
    stats = _lib.McStats()
    L.ufem_mc_get_stats(C.byref(stats))
    return d_u[:, :n].T.cpu().numpy(), d_st.cpu().numpy(), d_it.cpu().numpy(), d_out.cpu().numpy(), stats


def _mean_stiffness(m, ifld):
    """The oracle's K (supports applied) at the mean inputs, as a sparse matrix."""
    from oracle.oracle import OracleModel
    from test_mc_gpu import model_from_sample
    o = OracleModel(model_from_sample(m, ifld.mean(axis=0))).run_static()
    fp, dp, pos, dat = o["K_frompos"], o["K_defpos"], o["K_pos"], o["Kbc_data"]
    rows, cols, vals = [], [], []
    for i in range(len(fp)):
        for j in range(fp[i], fp[i] + dp[i]):
            if pos[j] <= 0:
                break
            rows.append(i)
            cols.append(pos[j] - 1)
            vals.append(dat[j])
    n = len(fp)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def _coarse_space(m, u, ifld, nmodes):
    U, _, _ = np.linalg.svd(u.T, full_matrices=False)
    phi = U[:, :nmodes]
    K = _mean_stiffness(m, ifld)
    E = phi.T @ (K @ phi)
    Lc = np.linalg.cholesky(0.5 * (E + E.T))
    return np.linalg.solve(Lc, phi.T).T  # Phi L^-T


@pytest.fixture(scope="module")
def beam():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    m = mg.warm_beam(24, 6, 6, zones=8)
    g = GpuModel(m)
    train = mg.warm_samples(m, 256, first_sample=0)
    ev = mg.warm_samples(m, 300, first_sample=1000)   # 3 groups, the last one partly padding
    u_train = _solve(g, train, coarse=0)[0]
    return m, g, train, ev, u_train


@pytest.mark.parametrize("nmodes", [16, 64, 128])
def test_coarse_solution_matches_jacobi(beam, nmodes):
    from ufem_b200.mc import set_coarse
    m, g, train, ev, u_train = beam
    set_coarse(g, None)
    u0, st0, it0, o0, s0 = _solve(g, ev)
    assert s0.coarse_modes == 0
    set_coarse(g, _coarse_space(m, u_train, train, nmodes))
    try:
        u1, st1, it1, o1, s1 = _solve(g, ev)
    finally:
        set_coarse(g, None)
    assert s1.coarse_modes == nmodes
    assert (st0 == 0).all() and (st1 == 0).all()
    assert np.abs(u1 - u0).max() <= 1e-6 * np.abs(u0).max()
    assert np.abs(o1 - o0).max() <= 1e-6 * np.abs(o0).max()
    # the leading modes (well above the snapshots' 1e-8 solve accuracy) take
    # the smooth modes off the Jacobi PCG.  128 modes of 256 snapshots of a
    # 9-input family reach the solver-noise modes, which the additive
    # correction lifts to the top of the spectrum: only the answer is checked.
    if nmodes <= 64:
        assert it1.mean() < 0.8 * it0.mean(), (nmodes, it0.mean(), it1.mean())


def test_coarse_run_twice_identical(beam):
    from ufem_b200.mc import set_coarse
    m, g, train, ev, u_train = beam
    set_coarse(g, _coarse_space(m, u_train, train, 32))
    try:
        a = _solve(g, ev)
        b = _solve(g, ev)
    finally:
        set_coarse(g, None)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])


def test_any_coarse_space_gives_the_same_answer(beam):
    """A poor coarse space (16 random directions, rows scaled to 0.3 D^-1/2
    so that M stays near the Jacobi preconditioner) leaves M SPD: the same
    solutions.  (Large random directions are SPD too, but make M so badly
    conditioned that the iteration cap ends the solves.)"""
    from ufem_b200.mc import set_coarse
    m, g, train, ev, u_train = beam
    rng = np.random.default_rng(5)
    d = _mean_stiffness(m, train).diagonal()
    R = rng.standard_normal((len(d), 16)) * (0.3 / np.sqrt(16.0 * d))[:, None]
    u0, st0, it0, _, _ = _solve(g, ev[:130], coarse=0)
    set_coarse(g, R)
    try:
        u1, st1, it1, _, s1 = _solve(g, ev[:130])
    finally:
        set_coarse(g, None)
    assert s1.coarse_modes == 16
    assert (st0 == 0).all() and (st1 == 0).all()
    assert np.abs(u1 - u0).max() <= 1e-6 * np.abs(u0).max()


def test_coarse_off_by_option_and_on_other_precisions(beam):
    """opt.coarse = 0 and precisions 0/1 ignore the model's coarse space."""
    from ufem_b200.mc import set_coarse
    m, g, train, ev, u_train = beam
    set_coarse(g, _coarse_space(m, u_train, train, 16))
    try:
        u0, _, it0, _, s0 = _solve(g, ev[:100], coarse=0)
        ua, _, ita, _, _ = _solve(g, ev[:100], coarse=0)
        for prec in (0, 1):
            _, st, _, _, sp_ = _solve(g, ev[:100], precision=prec)
            assert sp_.coarse_modes == 0 and (st == 0).all()
    finally:
        set_coarse(g, None)
    assert s0.coarse_modes == 0
    assert np.array_equal(u0, ua) and np.array_equal(it0, ita)


def test_multi_mesh_launch_with_and_without_coarse(beam):
    """One launch over a mesh with a coarse space and one without."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve, set_coarse
    m, g, train, ev, u_train = beam
    m2 = mg.warm_beam(10, 3, 3, zones=4)
    g2 = GpuModel(m2)
    f2 = mg.warm_samples(m2, 70, first_sample=50)
    ref, _ = mc_solve([g, g2], [ev[:150], f2], precision=2, coarse=0)
    set_coarse(g, _coarse_space(m, u_train, train, 32))
    try:
        res, stats = mc_solve([g, g2], [ev[:150], f2], precision=2)
    finally:
        set_coarse(g, None)
    assert stats.coarse_modes == 32
    for k in range(2):
        assert (res[k][1] == 0).all() and (ref[k][1] == 0).all()
        assert np.abs(res[k][0] - ref[k][0]).max() <= 1e-6 * np.abs(ref[k][0]).max()
    assert res[0][2].mean() < ref[0][2].mean()
    # the mesh without a coarse space runs Jacobi PCG as before; the launch
    # with a coarse space tiles the rows differently (512-thread blocks), so
    # its FP64 partial sums add in another order: at most one iteration apart
    assert np.abs(res[1][2] - ref[1][2]).max() <= 1


def test_set_coarse_rejects_bad_sizes(beam):
    from ufem_b200 import _lib
    m, g, train, ev, u_train = beam
    L = _lib.load()
    AF_ERR_VAL = -3
    assert L.ufem_mc_set_coarse(g.h, 17, None) == AF_ERR_VAL    # not a multiple of 16
    assert L.ufem_mc_set_coarse(g.h, 144, None) == AF_ERR_VAL   # above 128
    assert L.ufem_mc_set_coarse(g.h, 16, None) == AF_ERR_VAL    # no array
    assert L.ufem_mc_set_coarse(g.h, 0, None) == 0


def test_warm_start_sets_coarse_space():
    """Training sets the coarse space from the leading POD modes; the warm
    solve with it gives the same outputs as without, in fewer iterations."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.warm import WarmStart
    m = mg.warm_beam(24, 6, 6, zones=8)
    g = GpuModel(m)
    cols, logs, sc = mg.warm_features(m)
    ws = WarmStart(g, cols, logs, sc, n_modes=32, n_hidden=64, n_snapshots=256, epochs=20, batch=128,
                   n_coarse=32)
    ts = ws.train(mg.warm_samples(m, 512), precision=2)
    assert ts["coarse_modes"] in (16, 32)   # the modes above the energy floor, a multiple of 16
    ws.set_guess_mode(1)
    ev = mg.warm_samples(m, 200, first_sample=5000)
    o0, st0, it0, w0 = ws.solve(ev, precision=2, coarse=False)
    o1, st1, it1, w1 = ws.solve(ev, precision=2, coarse=True)
    assert (st0 == 0).all() and (st1 == 0).all()
    assert np.abs(o1 - o0).max() <= 1e-6 * np.abs(o0).max()
    assert it1.mean() < 0.8 * it0.mean(), (it0.mean(), it1.mean())


def test_warm_solve_sample_ordering_returns_callers_order():
    """ufem_warm_solve solves the samples sorted by the spread of log(E / mean
    E) and returns everything in the caller's order: against the same warm
    start without ordering (same seed, same basis), the outputs agree within
    1e-6 sample by sample and the per-sample iteration counts within 2 (the
    grouping changes only when a group's true-residual passes run)."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.warm import WarmStart
    m = mg.warm_beam(24, 6, 6, zones=8)
    g = GpuModel(m)
    cols, logs, sc = mg.warm_features(m)
    tr = mg.warm_samples(m, 512)
    ev = mg.warm_samples(m, 300, first_sample=7000)
    res = []
    for order in (0, 1):
        ws = WarmStart(g, cols, logs, sc, n_modes=32, n_hidden=64, n_snapshots=256, epochs=5, batch=128,
                       n_coarse=32, order_samples=order)
        ws.train(tr, precision=2)
        ws.set_guess_mode(1)
        res.append(ws.solve(ev, precision=2))
        del ws
    (o0, st0, it0, _), (o1, st1, it1, _) = res
    assert (st0 == 0).all() and (st1 == 0).all()
    assert (np.abs(o1 - o0).max(axis=1) <= 1e-6 * np.abs(o0).max(axis=1)).all()
    assert np.abs(it1 - it0).max() <= 2


def test_warm_solve_ordering_with_non_finite_samples():
    """Non-finite inputs sort last (their ordering score is not finite): they
    report UFEM_ST_NAN at their own positions, every other sample converges
    to the outputs it has in a batch without them."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import ST_NAN
    from ufem_b200.warm import WarmStart
    m = mg.warm_beam(24, 6, 6, zones=8)
    g = GpuModel(m)
    cols, logs, sc = mg.warm_features(m)
    ws = WarmStart(g, cols, logs, sc, n_modes=32, n_hidden=64, n_snapshots=256, epochs=5, batch=128, n_coarse=32)
    ws.train(mg.warm_samples(m, 512), precision=2)
    ws.set_guess_mode(1)
    ev = mg.warm_samples(m, 260, first_sample=3000)
    bad = [3, 140, 259]
    evb = ev.copy()
    evb[bad[0], 0] = np.nan          # an E
    evb[bad[1], 5] = np.inf          # another E
    evb[bad[2], len(m.mp_vals)] = np.nan  # the load factor
    o0, st0, it0, _ = ws.solve(ev, precision=2)
    o1, st1, it1, _ = ws.solve(evb, precision=2)
    good = np.setdiff1d(np.arange(ev.shape[0]), bad)
    assert (st0 == 0).all()
    assert (st1[bad] == ST_NAN).all() and (st1[good] == 0).all()
    assert (np.abs(o1[good] - o0[good]).max(axis=1) <= 1e-6 * np.abs(o0[good]).max(axis=1)).all()


def test_coarse_space_wider_than_the_guess_basis():
    """n_coarse > n_modes: the POD fit computes max(n_modes, n_coarse) modes,
    the guess and the MLP use the leading n_modes, the coarse space up to
    n_coarse (above the energy floor); the basis returned has n_modes
    columns, and the solve matches the one without a coarse space."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.warm import WarmStart
    m = mg.warm_beam(24, 6, 6, zones=8)
    g = GpuModel(m)
    cols, logs, sc = mg.warm_features(m)
    ws = WarmStart(g, cols, logs, sc, n_modes=32, n_hidden=64, n_snapshots=256, epochs=5, batch=128, n_coarse=64)
    ts = ws.train(mg.warm_samples(m, 512), precision=2)
    assert 32 < ts["coarse_modes"] <= 64
    phi, s2 = ws.basis()
    assert phi.shape[1] == 32 and np.abs(phi.T @ phi - np.eye(32)).max() < 1e-8
    ws.set_guess_mode(1)
    ev = mg.warm_samples(m, 200, first_sample=5000)
    o0, st0, it0, _ = ws.solve(ev, precision=2, coarse=False)
    o1, st1, it1, _ = ws.solve(ev, precision=2, coarse=True)
    assert (st0 == 0).all() and (st1 == 0).all()
    assert np.abs(o1 - o0).max() <= 1e-6 * np.abs(o0).max()
    assert it1.mean() < 0.8 * it0.mean()


def test_coarse_on_quads_and_two_coarse_meshes():
    """The coarse phases on the quad family (2x2 blocks, plane stress), and in
    one launch with two brick meshes that both carry a coarse space (one
    launch holds one element family): the same answers as the Jacobi-only
    solves."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve, set_coarse
    quad = mg.mc_attach_vars(mg.plate_quad(32, 8, 4.0, 1.0, distort=0.2, seed=3))
    fq = mg.mc_samples(quad, mesh_id=6, nsamp=150)
    gq = GpuModel(quad)
    b1, b2 = mg.warm_beam(16, 4, 4, zones=4), mg.warm_beam(24, 6, 6, zones=8)
    f1, f2 = mg.warm_samples(b1, 140, first_sample=300), mg.warm_samples(b2, 90, first_sample=700)
    g1, g2 = GpuModel(b1), GpuModel(b2)
    refq, _ = mc_solve([gq], [fq], precision=2, coarse=0)
    refb, _ = mc_solve([g1, g2], [f1, f2], precision=2, coarse=0)
    tq = mg.mc_samples(quad, mesh_id=7, nsamp=64)
    t1, t2 = mg.warm_samples(b1, 64), mg.warm_samples(b2, 128)
    set_coarse(gq, _coarse_space(quad, _solve(gq, tq, coarse=0)[0], tq, 16))
    set_coarse(g1, _coarse_space(b1, _solve(g1, t1, coarse=0)[0], t1, 16))
    set_coarse(g2, _coarse_space(b2, _solve(g2, t2, coarse=0)[0], t2, 32))
    try:
        resq, sq = mc_solve([gq], [fq], precision=2)
        resb, sb = mc_solve([g1, g2], [f1, f2], precision=2)
    finally:
        for g in (gq, g1, g2):
            set_coarse(g, None)
    assert sq.coarse_modes == 16 and sb.coarse_modes == 32
    for res, ref in ((resq, refq), (resb, refb)):
        for k in range(len(res)):
            assert (res[k][1] == 0).all() and (ref[k][1] == 0).all()
            assert np.abs(res[k][0] - ref[k][0]).max() <= 1e-6 * np.abs(ref[k][0]).max()


def test_precision4_without_a_guess_runs_in_precision3(beam):
    """FP32 SpMV products need a starting guess: a launch without one runs in
    precision 3 (same iterations and answer, bitwise), and converges with the
    coarse space where FP32 products from zero would not."""
    from ufem_b200.mc import set_coarse
    m, g, train, ev, u_train = beam
    set_coarse(g, _coarse_space(m, u_train, train, 32))
    try:
        u3, st3, it3, o3, _ = _solve(g, ev, precision=3)
        u4, st4, it4, o4, _ = _solve(g, ev, precision=4)
    finally:
        set_coarse(g, None)
    assert (st4 == 0).all()
    assert np.array_equal(u3, u4) and np.array_equal(it3, it4) and np.array_equal(o3, o4)
