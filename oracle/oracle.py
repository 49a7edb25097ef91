"""ctypes binding of the C oracle restatement (oracle/ufem_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker; the product never calls
it.  Build with ``make -f oracle/Makefile``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

AF_OK = 0
SOLVER_CGWJ, SOLVER_SSOR, SOLVER_BICG = 0, 1, 2
EPS_REF = 1e-17 / 10000.0   # FEM_ZERO/10000, fem/fem.h:59 and fem/fem_sol.c:1722

_l = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run make -f oracle/Makefile)")
        L = C.CDLL(path)
        L.orc_model_new.restype = C.c_void_p
        L.orc_model_new.argtypes = [C.c_long, _d, C.c_long, C.c_long, _l, _l, _l, _l,
                                    C.c_long, _l, _l, _d, C.c_long,
                                    C.c_long, _l, _l, _l, _d, C.c_long,
                                    C.c_long, _l, _l, _l, _d]
        L.orc_model_free.argtypes = [C.c_void_p]
        for fn in ("orc_fill_K", "orc_add_loads", "orc_add_disps"):
            getattr(L, fn).argtypes = [C.c_void_p]
        L.orc_dofs.argtypes = [C.c_void_p, C.POINTER(C.c_long)]
        L.orc_get_ndoffld.argtypes = [C.c_void_p, _l]
        L.orc_K_len.restype = C.c_long
        L.orc_K_len.argtypes = [C.c_void_p]
        L.orc_rows.restype = C.c_long
        L.orc_rows.argtypes = [C.c_void_p]
        L.orc_get_K.argtypes = [C.c_void_p, _l, _l, _l, _d]
        L.orc_get_F.argtypes = [C.c_void_p, _d]
        L.orc_get_u.argtypes = [C.c_void_p, _d]
        L.orc_set_u.argtypes = [C.c_void_p, _d]
        L.orc_solve.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_long, C.POINTER(C.c_long)]
        L.orc_results.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_strains.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_reac_len.restype = C.c_long
        L.orc_reac_len.argtypes = [C.c_void_p]
        L.orc_elem_ke.argtypes = [C.c_void_p, C.c_long, _d]
        L.orc_quad_ke.argtypes = [_d, C.c_double, C.c_double, C.c_double, _d]
        L.orc_brick_ke.argtypes = [_d, C.c_double, C.c_double, _d]
        for fn in ("orc_eqs_cgwj", "orc_eqs_cgwssor", "orc_eqs_bicgs"):
            getattr(L, fn).argtypes = [C.c_long, _l, _l, _l, _d, _d, _d, C.c_double, C.c_long,
                                       C.POINTER(C.c_long)]
        _LIB = L
    return _LIB


class OracleModel:
    """One model in the oracle, driven like femSolve (fem/fem_sol.c:1655)."""

    def __init__(self, model):
        L = lib()
        self.model = model
        rs_frm, rs_cnt, rs_vals = model.rs_flat()
        mp_frm, mp_cnt, mp_vals = model.mp_flat()
        self._keep = [np.ascontiguousarray(a) for a in (
            model.n_xyz.astype(np.float64), model.e_type, model.e_rs, model.e_mp,
            model.e_nodes.ravel(), rs_frm, rs_cnt, rs_vals.astype(np.float64) if len(rs_vals) else np.zeros(1),
            model.mp_type, mp_frm, mp_cnt, mp_vals, model.nl_node, model.nl_type, model.nl_dir,
            model.nl_val.astype(np.float64))]
        k = self._keep
        self.h = L.orc_model_new(model.nLen, k[0].ravel(), model.eLen, model.e_nodes.shape[1],
                                 k[1], k[2], k[3], k[4], len(model.rs_type), k[5], k[6], k[7],
                                 len(rs_vals), len(model.mp_type), k[8], k[9], k[10], k[11],
                                 len(mp_vals), len(model.nl_node), k[12], k[13], k[14], k[15])
        self.rows = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_model_free(self.h)
            self.h = None

    def dofs(self):
        n = C.c_long(0)
        rv = lib().orc_dofs(self.h, C.byref(n))
        if rv != AF_OK:
            raise RuntimeError(f"orc_dofs rv={rv}")
        self.rows = n.value
        out = np.zeros(self.model.nLen * 7, np.int64)
        lib().orc_get_ndoffld(self.h, out)
        return out

    def fill_K(self):
        rv = lib().orc_fill_K(self.h)
        if rv != AF_OK:
            raise RuntimeError(f"orc_fill_K rv={rv}")
        return self.get_K()

    def get_K(self):
        L = lib()
        n, ln = L.orc_rows(self.h), L.orc_K_len(self.h)
        fp, dp = np.zeros(n, np.int64), np.zeros(n, np.int64)
        pos, dat = np.zeros(ln, np.int64), np.zeros(ln, np.float64)
        L.orc_get_K(self.h, fp, dp, pos, dat)
        return fp, dp, pos, dat

    def get_F(self):
        F = np.zeros(self.rows, np.float64)
        lib().orc_get_F(self.h, F)
        return F

    def get_u(self):
        u = np.zeros(self.rows, np.float64)
        lib().orc_get_u(self.h, u)
        return u

    def loads_bcs(self):
        lib().orc_add_loads(self.h)
        F_loads = self.get_F()
        rv = lib().orc_add_disps(self.h)
        if rv != AF_OK:
            raise RuntimeError(f"orc_add_disps rv={rv}")
        return F_loads

    def solve(self, solver=SOLVER_CGWJ, eps=EPS_REF, max_it=None):
        it = C.c_long(0)
        rv = lib().orc_solve(self.h, solver, eps, self.rows if max_it is None else max_it, C.byref(it))
        return rv, it.value

    def results(self):
        L = lib()
        quad = int(self.model.e_type[0]) == 2
        nip, ns = (4, 3) if quad else (27, 6)
        sig = np.zeros(self.model.eLen * nip * ns, np.float64)
        fint = np.zeros(self.rows, np.float64)
        reac = np.zeros(max(1, L.orc_reac_len(self.h)), np.float64)
        rv = L.orc_results(self.h, sig.ctypes.data, fint.ctypes.data, reac.ctypes.data)
        if rv != AF_OK:
            raise RuntimeError(f"orc_results rv={rv}")
        return sig.reshape(self.model.eLen, nip, ns), fint, reac[:L.orc_reac_len(self.h)]

    def strains(self):
        """Strains B u_e at every integration point, laid out like the
        stresses of ``results``."""
        quad = int(self.model.e_type[0]) == 2
        nip, ns = (4, 3) if quad else (27, 6)
        eps = np.zeros(self.model.eLen * nip * ns, np.float64)
        rv = lib().orc_strains(self.h, eps.ctypes.data)
        if rv != AF_OK:
            raise RuntimeError(f"orc_strains rv={rv}")
        return eps.reshape(self.model.eLen, nip, ns)

    def elem_ke(self, e):
        sz = 8 if int(self.model.e_type[e]) == 2 else 24
        out = np.zeros(sz * sz, np.float64)
        rv = lib().orc_elem_ke(self.h, e, out)
        if rv != AF_OK:
            raise RuntimeError(f"orc_elem_ke rv={rv}")
        return out.reshape(sz, sz)

    def run_static(self, solver=SOLVER_CGWJ, eps=EPS_REF):
        """The whole femSolve sequence; returns a dict of every intermediate."""
        out = {"ndoffld": self.dofs()}
        fp, dp, pos, dat = self.fill_K()
        out.update(K_frompos=fp, K_defpos=dp, K_pos=pos, K_data=dat)
        out["F_loads"] = self.loads_bcs()
        out["Kbc_data"] = self.get_K()[3]
        out["F_bc"] = self.get_F()
        rv, it = self.solve(solver, eps)
        out.update(rv_solve=rv, iters=it, u=self.get_u())
        sig, fint, reac = self.results()
        out.update(sig=sig, fint=fint, reac=reac)
        return out


def solve_rowslot(which, frompos, defpos, pos, data, b, x0, eps=EPS_REF, max_it=None):
    """Run one of the oracle solvers on a reference row-slot matrix."""
    fn = {"cgwj": "orc_eqs_cgwj", "ssor": "orc_eqs_cgwssor", "bicg": "orc_eqs_bicgs"}[which]
    x = np.array(x0, dtype=np.float64, copy=True)
    it = C.c_long(0)
    rv = getattr(lib(), fn)(len(frompos), frompos, defpos, pos, data, np.ascontiguousarray(b, np.float64),
                            x, eps, len(frompos) if max_it is None else max_it, C.byref(it))
    return rv, x, it.value
