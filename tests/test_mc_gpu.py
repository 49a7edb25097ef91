"""Monte Carlo on the GPU: the plugin ABI against the reference's own
libfem.so outputs (golden fixture), and the batched solve against per-sample
FP64 solves and the oracle.

Tolerance: displacements and reactions within 1e-8 relative (the batched
solves stop at true relative residual 1e-8 in FP64; the comparison allows
the condition-number amplification seen on these beams, 1e-6 on u for the
residual-1e-8 solves)."""
import os
import tempfile

import numpy as np
import pytest

from golden_util import load, model_from

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def mc_fixture():
    from ufem_b200 import meshgen as mg
    z = load("mc_beam_4x2x2")
    m = model_from(z)
    d = tempfile.mkdtemp()
    path = os.path.join(d, "mc.fem")
    mg.write_fem(m, path)
    return z, m, path


def test_plugin_abi_matches_reference(mc_fixture):
    from ufem_b200.mc import MonteLib
    z, m, path = mc_fixture
    lib = MonteLib(path)
    try:
        assert lib.interface_type() == 2
        assert lib.ilen == int(z["mc_ilen"]) and lib.olen == int(z["mc_olen"])
        assert lib.ovar_names() == [str(s) for s in z["onames"]]
        nmat = len(z["inames"])
        assert lib.ivar_names()[:nmat] == [str(s) for s in z["inames"]]
        ref = z["ofld"]
        prev_reac = np.zeros(ref.shape[1])
        is_reac = np.array([n.startswith("REAC") for n in lib.ovar_names()])
        for s in range(ref.shape[0]):
            rv, out = lib.solution(z["ifld"][s])
            assert rv == 0
            # displacements: the reference's FP64 solve
            assert relerr(out[~is_reac], ref[s, ~is_reac]) <= 1e-8
            # reactions: the reference accumulates them across samples
            # (resRval is never cleared in monte_linear_solver); per sample
            # they are the difference of consecutive outputs
            ref_reac = ref[s, is_reac] - prev_reac[is_reac]
            prev_reac = ref[s]
            assert relerr(out[is_reac], ref_reac) <= 1e-8
    finally:
        lib.close()


def test_batch_matches_single_samples(mc_fixture):
    from ufem_b200.mc import MonteLib
    z, m, path = mc_fixture
    lib = MonteLib(path)
    try:
        rv, ob, st = lib.solution_batch(z["ifld"])
        assert rv == 0 and (st == 0).all()
        for s in range(z["ifld"].shape[0]):
            rv, o1 = lib.solution(z["ifld"][s])
            assert relerr(ob[s], o1) <= 1e-6
    finally:
        lib.close()


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_uneven_meshes_one_launch(precision):
    """Three meshes of uneven size and sample counts (not multiples of the
    sample group) in one launch, against per-sample FP64 oracle solves."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve
    from oracle.oracle import OracleModel
    specs = [(4, 1, 1, 37), (8, 2, 2, 150), (6, 3, 2, 70)]
    models, gms, iflds = [], [], []
    for k, (nx, ny, nz, ns) in enumerate(specs):
        m = mg.beam_brick(nx, ny, nz, 2.0 * nx / 4, 0.5 * ny, 0.5 * nz, per_element_material=True)
        mg.mc_attach_vars(m, n_out_nodes=3)
        models.append(m)
        gms.append(GpuModel(m))
        iflds.append(mg.mc_samples(m, mesh_id=k, nsamp=ns))
    res, stats = mc_solve(gms, iflds, precision=precision, tol=1e-8)
    for k, m in enumerate(models):
        ofld, st, it = res[k]
        assert (st == 0).all(), (k, st)
        assert (it > 0).all()
        for s in (0, iflds[k].shape[0] // 2, iflds[k].shape[0] - 1):
            mm = model_from_sample(m, iflds[k][s])
            om = OracleModel(mm)
            o = om.run_static()
            # RES_D outputs = u at the chosen tip nodes
            rows = []
            nd = o["ndoffld"]
            for row in m.mc_vars[m.mc_ilen:]:
                if row[1] == mg.MONTE_VTYPE_RES_D:
                    rows.append(nd[row[2] * 7 + row[3] - 1] - 1)
            assert relerr(ofld[s, :len(rows)], o["u"][rows]) <= 1e-6
            reac = o["reac"]
            reac_idx = [j for j, row in enumerate(m.mc_vars[m.mc_ilen:]) if row[1] == mg.MONTE_VTYPE_RES_R]
            # reaction outputs: first support node, UX and UZ
            rlist = list(zip(o_reac_nodes(m), o_reac_dofs(m)))
            for j in reac_idx:
                row = m.mc_vars[m.mc_ilen + j]
                r = rlist.index((row[2], row[3]))
                assert abs(ofld[s, j] - reac[r]) <= 1e-6 * np.abs(reac).max()
    assert stats.pcg_iterations > 0


def o_reac_nodes(m):
    return [int(n) for n, t, v in zip(m.nl_node, m.nl_type, m.nl_val) if t == 1 and v == 0.0]


def o_reac_dofs(m):
    return [int(d) for d, t, v in zip(m.nl_dir, m.nl_type, m.nl_val) if t == 1 and v == 0.0]


def model_from_sample(m, row):
    """The model with one MC sample's inputs applied (E per material, forces)."""
    import copy
    from ufem_b200 import meshgen as mg
    mm = copy.deepcopy(m)
    mm.mp_vals = [v.copy() for v in m.mp_vals]
    mm.nl_val = m.nl_val.copy()
    for var in m.mc_vars[:m.mc_ilen]:
        pos, ty, item, sub, it = [int(x) for x in var]
        if ty == mg.MONTE_VTYPE_MAT and sub == mg.MAT_EX:
            mm.mp_vals[item][1] = row[pos]
        elif ty == mg.MONTE_VTYPE_NLD:
            for j in range(len(mm.nl_node)):
                if mm.nl_node[j] == item and mm.nl_type[j] == sub and mm.nl_dir[j] == it:
                    mm.nl_val[j] = row[pos]
                    break
    return mm


def test_zero_load_sample_converges_at_once():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve
    m = mg.beam_brick(4, 2, 2, 2.0, 1.0, 1.0, per_element_material=True)
    mg.mc_attach_vars(m)
    f = mg.mc_samples(m, 5, 3)
    f[1, len(m.mp_vals):] = 0.0          # sample 1: no load
    res, _ = mc_solve([GpuModel(m)], [f])
    ofld, st, it = res[0]
    assert (st == 0).all()
    assert it[1] == 0 and not ofld[1].any()
    assert it[0] > 0 and it[2] > 0


def test_batched_run_twice_identical():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve
    m = mg.beam_brick(6, 2, 2, 3.0, 1.0, 1.0, per_element_material=True)
    mg.mc_attach_vars(m)
    f = mg.mc_samples(m, 9, 200)
    g = GpuModel(m)
    a, _ = mc_solve([g], [f])
    b, _ = mc_solve([g], [f])
    assert np.array_equal(a[0][0], b[0][0]) and np.array_equal(a[0][2], b[0][2])


def test_iteration_cap_reports_maxit():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import ST_MAXIT, mc_solve
    m = mg.beam_brick(8, 2, 2, 4.0, 1.0, 1.0, per_element_material=True)
    mg.mc_attach_vars(m)
    f = mg.mc_samples(m, 3, 5)
    res, _ = mc_solve([GpuModel(m)], [f], max_iters=3)
    assert (res[0][1] == ST_MAXIT).all()


def _solve_u(g, ifld, precision):
    """Batched solve through ufem_mc_solve_device: (u [nsamp][ndof], status, iters)."""
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
    d_u = torch.zeros((g.ndof, S), dtype=torch.float64, device="cuda")
    vp = lambda t: (C.c_void_p * 1)(t.data_ptr())
    opt = default_options()
    opt.precision = precision
    rv = L.ufem_mc_solve_device(1, (C.c_void_p * 1)(g.h.value), np.array([n], np.int64).ctypes.data_as(
        C.POINTER(C.c_long)), vp(d_in), vp(d_out), vp(d_st), vp(d_it), (C.c_void_p * 1)(), vp(d_u), C.byref(opt))
    _lib.check("ufem_mc_solve_device", rv)
    return d_u[:, :n].T.cpu().numpy(), d_st.cpu().numpy(), d_it.cpu().numpy(), d_out.cpu().numpy()


def _drop_first_input(m, ifld):
    """The model with its first Monte Carlo input (material 0's E) made
    non-random, and the inputs without that column."""
    rows = [r.copy() for r in m.mc_vars]
    ins = rows[1:m.mc_ilen]
    outs = rows[m.mc_ilen:]
    for j, r in enumerate(ins):
        r[0] = j
    m.mc_vars = np.array(ins + outs, dtype=np.int64)
    m.mc_ilen -= 1
    return ifld[:, 1:].copy()


def _implicit_cases():
    from ufem_b200 import meshgen as mg
    zones = mg.warm_beam(12, 3, 3, zones=4)
    f_zones = mg.warm_samples(zones, 100)
    part = mg.mc_attach_vars(mg.beam_brick(6, 2, 2, 3.0, 1.0, 1.0, zones=3))
    f_part = _drop_first_input(part, mg.mc_samples(part, mesh_id=4, nsamp=70))
    quad = mg.mc_attach_vars(mg.plate_quad(16, 4, 4.0, 1.0, distort=0.2, seed=3))
    f_quad = mg.mc_samples(quad, mesh_id=6, nsamp=50)
    elem = mg.mc_attach_vars(mg.beam_brick(5, 2, 2, 2.5, 1.0, 1.0, per_element_material=True))
    f_elem = mg.mc_samples(elem, mesh_id=7, nsamp=40)
    return [("zones", zones, f_zones), ("constant_part", part, f_part), ("quad", quad, f_quad),
            ("per_element", elem, f_elem)]


@pytest.mark.parametrize("case", range(4))
def test_implicit_form_matches_explicit_fp64(case):
    """precision 2 (each block formed inside the PCG kernel from the shared
    unit-E element blocks summed per random multiplier) against precision 0
    (an explicit FP64 matrix per sample): E zones (several elements per
    multiplier), a non-random material (the constant part), quads (B = 2)
    and per-element E.  Both are FP64 PCGs to the true relative residual
    1e-8: solutions within 1e-6 relative, iteration counts within 3 %."""
    from ufem_b200.api import GpuModel
    name, m, f = _implicit_cases()[case]
    g = GpuModel(m)
    u0, st0, it0, o0 = _solve_u(g, f, 0)
    u2, st2, it2, o2 = _solve_u(g, f, 2)
    assert (st0 == 0).all() and (st2 == 0).all(), name
    assert np.abs(u2 - u0).max() <= 1e-6 * np.abs(u0).max(), name
    assert np.abs(o2 - o0).max() <= 1e-6 * max(np.abs(o0).max(), 1e-300), name
    assert (np.abs(it2 - it0) <= 0.03 * it0 + 2).all(), (name, it0, it2)


def test_implicit_run_twice_identical():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    m = mg.warm_beam(8, 2, 2, zones=4)
    f = mg.warm_samples(m, 150)
    g = GpuModel(m)
    a = _solve_u(g, f, 2)
    b = _solve_u(g, f, 2)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])


def test_autotune_writes_cache_and_is_used(tmp_path):
    """The autotuner times every candidate launch shape on the batch, writes
    its choice to the cache file and later solves that leave the shape at 0
    use it; the solution agrees across shapes within the batched tolerance."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import autotune, mc_solve
    m = mg.warm_beam(8, 2, 2, zones=4)
    f = mg.warm_samples(m, 200)
    g = GpuModel(m)
    cache = tmp_path / "tune.txt"
    best = autotune([g], [f], precision=2, cache_path=str(cache))
    assert best.tiles_per_block in (3, 6, 12, 24, 48) and best.unroll in (2, 4, 8)
    line = cache.read_text().split()
    assert len(line) == 5 and line[0].endswith(f"/p2/b3/{g.bsr_shape()[1]}x256")
    assert int(line[1]) == best.tiles_per_block and int(line[2]) == best.unroll
    assert int(line[3]) == best.lane_samples in (2, 4)
    res, st = mc_solve([g], [f], precision=2)
    o_t, s_t, _ = res[0]
    assert st.tiles_per_block == best.tiles_per_block and st.unroll == best.unroll
    assert st.lane_samples == best.lane_samples
    res, _ = mc_solve([g], [f], precision=2, tiles_per_block=3, unroll=2)
    o_f, s_f, _ = res[0]
    assert (s_t == 0).all() and (s_f == 0).all()
    # the tile count changes the grouping of the dot products, not the answer
    assert np.abs(o_t - o_f).max() <= 1e-6 * np.abs(o_f).max()


@pytest.mark.parametrize("precision", [1, 2])
def test_non_finite_samples_report_nan_and_leave_others_alone(precision):
    """A sample with a NaN E value or a NaN load is reported UFEM_ST_NAN (not
    converged, not a breakdown); the other samples of its group converge to
    the same outputs as without it."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import ST_NAN, mc_solve
    m = mg.warm_beam(6, 2, 2, zones=3)
    f = mg.warm_samples(m, 20)
    g = GpuModel(m)
    (o_ok, s_ok, _), = mc_solve([g], [f], precision=precision)[0]
    bad = f.copy()
    bad[3, 0] = np.nan                  # E of zone 0
    bad[7, len(m.mp_vals)] = np.nan     # one tip force
    (o_b, s_b, _), = mc_solve([g], [bad], precision=precision)[0]
    assert s_b[3] == ST_NAN and s_b[7] == ST_NAN
    keep = np.setdiff1d(np.arange(20), [3, 7])
    assert (s_b[keep] == 0).all() and (s_ok == 0).all()
    assert np.abs(o_b[keep] - o_ok[keep]).max() <= 1e-12 * np.abs(o_ok).max()


def test_mesh_without_samples_in_a_multi_mesh_launch():
    """One mesh of a launch has no samples: the others solve as usual."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve
    a = mg.warm_beam(6, 2, 2, zones=3)
    b = mg.warm_beam(4, 2, 2, zones=2)
    fa = mg.warm_samples(a, 30)
    fb = mg.warm_samples(b, 0)
    for prec in (1, 2):
        res, _ = mc_solve([GpuModel(a), GpuModel(b)], [fa, fb], precision=prec)
        assert (res[0][1] == 0).all() and res[1][1].shape == (0,)
