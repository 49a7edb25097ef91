"""Generate the golden fixtures in tests/golden/ by running the reference.

The reference uFEM solver has no golden vectors or known-answer tests of its
own, so the fixtures come from the reference implementation itself: its C
sources are built unmodified by ``oracle/Makefile.ref`` into
``oracle/_ref/serial/`` and driven by ``oracle/ref_harness.c`` (the femSolve
sequence, fem/fem_sol.c:1655-1760) and, for the Monte Carlo plugin ABI, by
loading ``oracle/_ref/serial/libfem_ref.so`` and calling ``monte_init_lib_stuff``
/ ``monte_solution`` (fem/fem_mont.c:424, :694) as an external driver would.

Run it in a container that has the reference sources (it builds them if
needed):

    python tests/golden/make_golden.py             # every fixture
    python tests/golden/make_golden.py mc_outputs  # the Monte Carlo output fixtures only
    python tests/golden/make_golden.py beam_80x20x20  # config 2's displacements only

The fixtures are committed; tests only read them.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from ufem_b200 import meshgen as mg  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "tests"))
from golden_util import model_sha  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref", "serial")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def build_ref():
    if not os.path.exists(os.path.join(REF_DIR, "ref_harness")):
        subprocess.check_call(["make", "-f", os.path.join(ROOT, "oracle", "Makefile.ref"), "-j8"], cwd=ROOT)


def run_harness(model: mg.Model, solver="cgwj", want_ke=True) -> dict:
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "in.fem")
        mg.write_fem(model, inp)
        args = [os.path.join(REF_DIR, "ref_harness"), inp, d, "-s", solver]
        if want_ke:
            args.append("--ke")
        subprocess.run(args, check=False, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        meta = json.load(open(os.path.join(d, "meta.json")))
        out = {"meta": meta}
        for name in os.listdir(d):
            if name.endswith(".i64"):
                out[name[:-4]] = np.fromfile(os.path.join(d, name), dtype=np.int64)
            elif name.endswith(".f64"):
                out[name[:-4]] = np.fromfile(os.path.join(d, name), dtype=np.float64)
        return out


def model_arrays(model: mg.Model) -> dict:
    """The model tables, so tests can rebuild the model without the generator."""
    rs_frm, rs_cnt, rs_vals = model.rs_flat()
    mp_frm, mp_cnt, mp_vals = model.mp_flat()
    return dict(m_xyz=model.n_xyz, m_etype=model.e_type, m_ers=model.e_rs, m_emp=model.e_mp,
                m_enodes=model.e_nodes, m_rstype=model.rs_type, m_rscnt=rs_cnt, m_rsvals=rs_vals,
                m_mptype=model.mp_type, m_mpcnt=mp_cnt, m_mpvals=mp_vals, m_nlnode=model.nl_node,
                m_nltype=model.nl_type, m_nldir=model.nl_dir, m_nlval=model.nl_val)


def save_case(name: str, model: mg.Model, full: bool, ke_elems=None, solvers=("cgwj",)):
    res = run_harness(model, solvers[0], want_ke=True)
    nip, ns = (4, 3) if int(model.e_type[0]) == mg.ELEM_QUAD else (27, 6)
    sz = 8 if nip == 4 else 24
    out = model_arrays(model)
    out["meta"] = json.dumps(res["meta"])
    out["rv_solve"] = np.int64(res["meta"]["rv_solve"])
    out["ndoffld"] = res["ndoffld"]
    out["K_frompos"] = res["K_frompos"]
    out["K_defpos"] = res["K_defpos"]
    out["K_pos"] = res["K_pos"]
    ke = res["Ke"].reshape(model.eLen, sz, sz)
    out["u"] = res["u"]
    out["F_bc"] = res["F_bc"]
    out["F_loads"] = res["F_loads"]
    out["reac_node"], out["reac_dof"], out["reac_val"] = res["reac_node"], res["reac_dof"], res["reac_val"]
    out["eres"] = res["eres"].reshape(model.eLen, nip, ns)
    out["sha_K_data"] = sha(res["K_data"])
    out["sha_Kbc_data"] = sha(res["Kbc_data"])
    out["sha_Ke"] = sha(res["Ke"])
    if full:
        out["K_data"] = res["K_data"]
        out["Kbc_data"] = res["Kbc_data"]
        out["Ke"] = ke
    else:
        idx = np.asarray(ke_elems if ke_elems is not None else [0, model.eLen // 2, model.eLen - 1])
        out["Ke_idx"] = idx
        out["Ke"] = ke[idx]
    for s in solvers[1:]:
        r2 = run_harness(model, s, want_ke=False)
        out[f"u_{s}"] = r2["u"]
        out[f"rv_{s}"] = np.int64(r2["meta"]["rv_solve"])
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {os.path.getsize(path) / 1024:.0f} KiB, nDOFAct={res['meta']['nDOFAct']}")


MC_DRIVER = r"""
import ctypes as C, sys, numpy as np
lib = C.CDLL(sys.argv[1])
param = sys.argv[2].encode()
lib.monte_init_lib_stuff.argtypes = [C.c_char_p]
lib.monte_solution.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_long]
lib.monte_nums_of_vars.argtypes = [C.c_char_p, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_long)]
lib.monte_ivar_name.restype = C.c_char_p
lib.monte_ivar_name.argtypes = [C.c_char_p, C.c_long]
lib.monte_ovar_name.restype = C.c_char_p
lib.monte_ovar_name.argtypes = [C.c_char_p, C.c_long]
assert lib.monte_dlib_interface_type() == 2
assert lib.monte_init_lib_stuff(param) == 0
il, ol, ff = C.c_long(), C.c_long(), C.c_long()
lib.monte_nums_of_vars(param, C.byref(il), C.byref(ol), C.byref(ff))
ifld = np.load(sys.argv[3])
ofld = np.zeros((ifld.shape[0], ol.value))
rvs = []
for s in range(ifld.shape[0]):
    row = np.ascontiguousarray(ifld[s])
    out = np.zeros(ol.value)
    rvs.append(lib.monte_solution(param, row.ctypes.data, out.ctypes.data, 0))
    ofld[s] = out
# only the material inputs are named here: for NLD inputs monte_ivar_name
# indexes nlNode[] with the item (a node position, fem/fem_mont.c:203) while
# monte_solution matches the item against nlNode[j] (fem/fem_mont.c:757), so
# asking for those names reads past nlNode on this model.
nmat = int(sys.argv[5])
inames = [lib.monte_ivar_name(param, i).decode() for i in range(nmat)]
onames = [lib.monte_ovar_name(param, i).decode() for i in range(ol.value)]
np.savez(sys.argv[4], ofld=ofld, rv=np.array(rvs), ilen=il.value, olen=ol.value, ffunc=ff.value,
         inames=np.array(inames), onames=np.array(onames))
"""


def save_mc_case(name: str, model: mg.Model, nsamp: int):
    mg.mc_attach_vars(model, n_out_nodes=3)
    ifld = mg.mc_samples(model, mesh_id=99, nsamp=nsamp)
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "mc.fem")
        mg.write_fem(model, inp)
        np.save(os.path.join(d, "ifld.npy"), ifld)
        drv = os.path.join(d, "drv.py")
        open(drv, "w").write(MC_DRIVER)
        subprocess.run([sys.executable, drv, os.path.join(REF_DIR, "libfem_ref.so"), inp,
                        os.path.join(d, "ifld.npy"), os.path.join(d, "out.npz"), str(len(model.mp_vals))],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        r = np.load(os.path.join(d, "out.npz"))
        out = model_arrays(model)
        out.update(mc_vars=model.mc_vars, mc_ilen=model.mc_ilen, mc_olen=model.mc_olen, ifld=ifld,
                   ofld=r["ofld"], rv=r["rv"], inames=r["inames"], onames=r["onames"], ffunc=r["ffunc"])
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {os.path.getsize(path) / 1024:.0f} KiB, rv={r['rv'].tolist()}")


def _strength_materials(model: mg.Model, groups: np.ndarray, fy=20e6) -> mg.Model:
    """Give element e material record groups[e], each of type 5 (DENS, EX,
    NU, G, F_YC, F_YT, F_UC, F_UT; fem/fem_m005.c:39)."""
    ng = int(groups.max()) + 1
    model.e_mp = groups.astype(np.int64)
    model.mp_type = np.full(ng, mg.MAT_STRENGTH, np.int64)
    model.mp_vals = [np.array([2500.0, 30e9, 0.2, 12.5e9, fy, 2e6, 30e6, 2e6]) for _ in range(ng)]
    return model


def _scales(model: mg.Model):
    """Largest von Mises stress and |u| of the model as it stands (oracle)."""
    from oracle.oracle import OracleModel, SOLVER_SSOR
    r = OracleModel(model).run_static(SOLVER_SSOR)
    s = r["sig"]
    if s.shape[-1] == 3:
        j2 = ((s[..., 0] - s[..., 1]) ** 2 + s[..., 0] ** 2 + s[..., 1] ** 2) / 6 + s[..., 2] ** 2
    else:
        j2 = (((s[..., 0] - s[..., 1]) ** 2 + (s[..., 1] - s[..., 2]) ** 2 + (s[..., 2] - s[..., 0]) ** 2) / 6
              + (s[..., 3:] ** 2).sum(-1))
    return float(np.sqrt(3 * j2).max()), float(np.abs(r["u"]).max())


def save_mc_outputs_case(name: str, model: mg.Model, nsamp: int):
    """Every linear-static output of monte_fill_ofld_data and the failure
    function, from the reference libfem.so as an external driver calls it."""
    mg.mc_attach_outputs(model)
    vm, umax = _scales(model)
    # the max-displacement test compares sqrt(max |u|) with MAX_D
    # (femVecMaxAbs returns the square root, fem/fem_math.c:2163)
    ifld = mg.mc_outputs_samples(model, nsamp, vm_scale=vm, u_scale=float(np.sqrt(umax)))
    nmat = int(np.sum(model.mc_vars[:model.mc_ilen, 1] == mg.MONTE_VTYPE_MAT))
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "mc.fem")
        mg.write_fem(model, inp)
        np.save(os.path.join(d, "ifld.npy"), ifld)
        drv = os.path.join(d, "drv.py")
        open(drv, "w").write(MC_DRIVER)
        subprocess.run([sys.executable, drv, os.path.join(REF_DIR, "libfem_ref.so"), inp,
                        os.path.join(d, "ifld.npy"), os.path.join(d, "out.npz"), str(nmat)],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        r = np.load(os.path.join(d, "out.npz"))
        out = model_arrays(model)
        out.update(mc_vars=model.mc_vars, mc_ilen=model.mc_ilen, mc_olen=model.mc_olen, ifld=ifld,
                   ofld=r["ofld"], rv=r["rv"], inames=r["inames"], onames=r["onames"], ffunc=r["ffunc"])
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {os.path.getsize(path) / 1024:.0f} KiB, rv={r['rv'].tolist()}, ffunc={int(r['ffunc'])}")


def mc_outputs_cases():
    """The Monte Carlo output fixtures (type-5 materials with F_YC, mixed
    brick types 9/10, and a type-1 plate whose F_YC reads 0)."""
    m = mg.plate_quad(6, 3, 1.5, 0.75)
    _strength_materials(m, (np.arange(m.eLen) % 6 >= 3).astype(np.int64))
    save_mc_outputs_case("mc_out_plate_6x3", m, 8)
    b = mg.beam_brick(4, 2, 2, 2.0, 1.0, 1.0)
    ix = np.arange(b.eLen) % 4
    _strength_materials(b, (ix >= 2).astype(np.int64))
    b.e_type = np.where(ix >= 2, mg.ELEM_BRICK_W, mg.ELEM_BRICK).astype(np.int64)
    b.e_rs = (ix >= 2).astype(np.int64)
    b.rs_type = np.array([mg.ELEM_BRICK, mg.ELEM_BRICK_W], np.int64)
    b.rs_vals = [np.zeros(0), np.array([0.0])]
    save_mc_outputs_case("mc_out_beam_4x2x2", b, 8)
    save_mc_outputs_case("mc_out_plate_iso_4x2", mg.plate_quad(4, 2, 1.0, 0.5), 3)


def beam_80x20x20_case():
    """Config 2, the 80x20x20 brick cantilever (107,163 DOFs): the reference's
    displacements from its own femEqsCGwJ with its stopping rule (about a
    minute on one core).  Only u, the DOF map's hash and the model's hash are
    kept (the tables are regenerated by ``mg.beam_brick(80, 20, 20, 8.0, 2.0,
    2.0)``); u is stored with its last 12 mantissa bits cleared (relative
    rounding below 2.3e-13), which keeps the file small."""
    model = mg.beam_brick(80, 20, 20, 8.0, 2.0, 2.0)
    res = run_harness(model, "cgwj", want_ke=False)
    u = np.ascontiguousarray(res["u"], np.float64)
    uq = (u.view(np.uint64) & ~np.uint64(0xFFF)).view(np.float64)
    np.savez_compressed(os.path.join(HERE, "beam_80x20x20.npz"), u=uq, model_sha=model_sha(model),
                        ndoffld_sha=sha(res["ndoffld"].astype(np.int64)), rv_solve=res["meta"]["rv_solve"],
                        t_solve=res["meta"]["t_solve"])


def main():
    build_ref()
    if sys.argv[1:] == ["mc_outputs"]:
        mc_outputs_cases()
        return
    if sys.argv[1:] == ["beam_80x20x20"]:
        beam_80x20x20_case()
        return
    # config 1: the 64x16 cantilever plate (plane stress), 2,210 DOFs
    save_case("plate_64x16", mg.plate_quad(), full=False, ke_elems=[0, 1, 15, 16, 500, 1023])
    # distorted quads (non-rectangular Jacobians), full dumps, three solvers
    save_case("plate_6x3_distorted", mg.plate_quad(6, 3, 1.5, 0.75, distort=0.3, seed=3), full=True,
              solvers=("cgwj", "ssor", "bicg"))
    # plane strain (thickness 0 selects it, fem/fem_e002.c:400-407)
    save_case("plate_4x2_strain", mg.plate_quad(4, 2, 1.0, 0.5, thick=0.0, nu=0.3), full=True)
    # a nonzero prescribed displacement (femApplyDisp's Val != 0 branch)
    m = mg.plate_quad(4, 2, 1.0, 0.5)
    m.nl_val = m.nl_val.copy()
    m.nl_val[1] = 1e-4          # node 0, UY = 1e-4 m
    save_case("plate_4x2_prescribed", m, full=True)
    # distorted bricks, full dumps, three solvers
    save_case("brick_3x2x2_distorted", mg.beam_brick(3, 2, 2, 1.5, 1.0, 1.0, distort=0.25, seed=5),
              full=True, solvers=("cgwj", "ssor", "bicg"))
    # config 4a: the 20x5x5 Monte Carlo beam, 2,268 DOFs
    save_case("beam_20x5x5", mg.beam_brick(20, 5, 5, 8.0, 2.0, 2.0), full=False,
              ke_elems=[0, 1, 20, 100, 499])
    # the Monte Carlo plugin ABI: per-element E and a random end load
    save_mc_case("mc_beam_4x2x2", mg.beam_brick(4, 2, 2, 2.0, 1.0, 1.0, per_element_material=True), 4)
    mc_outputs_cases()
    beam_80x20x20_case()


if __name__ == "__main__":
    main()
