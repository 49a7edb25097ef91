"""Python mirror of the reference's solver interface over libufem_gpu.so.

``GpuModel`` follows femSolve (fem/fem_sol.c:1655-1760) step by step --
``fill_K(0)``, ``add_loads``, ``add_disps``, ``solve``, ``fill_K(1)`` -- with
the reference's return codes turned into :class:`ufem_b200._lib.UfemError`.
Every method calls the CUDA library; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .meshgen import Model

SOLVER_CGWJ, SOLVER_SSOR, SOLVER_BICG, SOLVER_CGWJ_MIXED = 0, 1, 2, 3
STOP_REFERENCE, STOP_RELRES = 0, 1
EPS_REF = 1e-17 / 10000.0   # FEM_ZERO/10000, fem/fem.h:59, fem/fem_sol.c:1722


def _lp(a):
    return a.ctypes.data_as(C.POINTER(C.c_long))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def tables_of(model: Model):
    """ufem_tables for ``model`` plus the arrays that keep it alive."""
    rs_frm, rs_cnt, rs_vals = model.rs_flat()
    mp_frm, mp_cnt, mp_vals = model.mp_flat()
    keep = dict(
        x=np.ascontiguousarray(model.n_xyz[:, 0], np.float64),
        y=np.ascontiguousarray(model.n_xyz[:, 1], np.float64),
        z=np.ascontiguousarray(model.n_xyz[:, 2], np.float64),
        et=np.ascontiguousarray(model.e_type, np.int64),
        ers=np.ascontiguousarray(model.e_rs, np.int64),
        emp=np.ascontiguousarray(model.e_mp, np.int64),
        efrom=np.ascontiguousarray(model.e_from(), np.int64),
        en=np.ascontiguousarray(model.e_nodes.ravel(), np.int64),
        rst=np.ascontiguousarray(model.rs_type, np.int64),
        rsf=np.ascontiguousarray(rs_frm, np.int64),
        rsv=np.ascontiguousarray(rs_vals if len(rs_vals) else np.zeros(1), np.float64),
        mpt=np.ascontiguousarray(model.mp_type, np.int64),
        mpf=np.ascontiguousarray(mp_frm, np.int64),
        mpv=np.ascontiguousarray(mp_vals, np.float64),
        nln=np.ascontiguousarray(model.nl_node, np.int64),
        nlt=np.ascontiguousarray(model.nl_type, np.int64),
        nld=np.ascontiguousarray(model.nl_dir, np.int64),
        nlv=np.ascontiguousarray(model.nl_val, np.float64),
    )
    k = keep
    t = _lib.Tables(
        model.nLen, _dp(k["x"]), _dp(k["y"]), _dp(k["z"]),
        model.eLen, _lp(k["et"]), _lp(k["ers"]), _lp(k["emp"]), _lp(k["efrom"]), _lp(k["en"]),
        len(model.rs_type), _lp(k["rst"]), _lp(k["rsf"]), len(rs_vals), _dp(k["rsv"]),
        len(model.mp_type), _lp(k["mpt"]), _lp(k["mpf"]), len(mp_vals), _dp(k["mpv"]),
        len(model.nl_node), _lp(k["nln"]), _lp(k["nlt"]), _lp(k["nld"]), _dp(k["nlv"]))
    return t, keep


def convert_input(text_path: str, bin_path: str) -> None:
    """Write the binary form of an input file (``ufem_convert_input``); host
    only.  ``GpuModel(path=...)`` and the Monte Carlo plugin read either form."""
    _lib.check("ufem_convert_input", _lib.load().ufem_convert_input(text_path.encode(), bin_path.encode()))


class GpuModel:
    """One model on the GPU (``ufem_model`` handle)."""

    def __init__(self, model: Model | None = None, path: str | None = None):
        L = _lib.load()
        h = C.c_void_p()
        self.model = model
        if path is not None:
            _lib.check("ufem_read_input", L.ufem_read_input(path.encode(), C.byref(h)))
        else:
            t, self._keep = tables_of(model)
            _lib.check("ufem_model_create", L.ufem_model_create(C.byref(t), C.byref(h)))
        self.h = h
        if model is not None and model.mc_vars is not None and model.mc_ilen > 0:
            self.set_mc_vars(model.mc_ilen, model.mc_olen, model.mc_vars)

    def set_mc_vars(self, ilen: int, olen: int, table):
        """Attach a Monte Carlo variable table (rows: pos, type, item, sub, iter)."""
        v = np.ascontiguousarray(np.asarray(table, np.int64).ravel())
        _lib.check("ufem_model_set_mc_vars", _lib.load().ufem_model_set_mc_vars(self.h, ilen, olen, _lp(v)))

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            _lib.load().ufem_model_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- shapes and patterns -------------------------------------------------
    @property
    def ndof(self) -> int:
        return _lib.load().ufem_ndof(self.h)

    def bsr_shape(self):
        b, nbr, nnzb = C.c_long(), C.c_long(), C.c_long()
        _lib.load().ufem_bsr_shape(self.h, C.byref(b), C.byref(nbr), C.byref(nnzb))
        return b.value, nbr.value, nnzb.value

    def ndoffld(self, nlen: int) -> np.ndarray:
        out = np.zeros(nlen * 7, np.int64)
        _lib.check("ufem_get_ndoffld", _lib.load().ufem_get_ndoffld(self.h, _lp(out)))
        return out

    def rowslot(self):
        L = _lib.load()
        n = self.ndof
        ln = C.c_long()
        _lib.check("ufem_export_rowslot", L.ufem_export_rowslot(self.h, None, None, None, C.byref(ln)))
        fp, dp, pos = np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(ln.value, np.int64)
        _lib.check("ufem_export_rowslot", L.ufem_export_rowslot(self.h, _lp(fp), _lp(dp), _lp(pos), C.byref(ln)))
        return fp, dp, pos

    def bsr_pattern(self):
        b, nbr, nnzb = self.bsr_shape()
        rp, ci = np.zeros(nbr + 1, np.int32), np.zeros(nnzb, np.int32)
        _lib.check("ufem_get_bsr_pattern", _lib.load().ufem_get_bsr_pattern(self.h, _ip(rp), _ip(ci)))
        return rp, ci

    @property
    def colours(self) -> int:
        return _lib.load().ufem_num_colours(self.h)

    def element_colours(self, n_elements: int | None = None):
        """Colour of each element (a model read from a file needs its element count)."""
        col = np.zeros(n_elements if n_elements is not None else self.model.eLen, np.int32)
        _lib.check("ufem_get_element_colours", _lib.load().ufem_get_element_colours(self.h, _ip(col)))
        return col

    # ---- the femSolve steps ----------------------------------------------------
    def fill_K(self, mode: int = 0):
        _lib.check("ufem_fill_K", _lib.load().ufem_fill_K(self.h, mode))

    def add_loads(self):
        _lib.check("ufem_add_loads", _lib.load().ufem_add_loads(self.h))

    def add_disps(self):
        _lib.check("ufem_add_disps", _lib.load().ufem_add_disps(self.h))

    def solve(self, solver=SOLVER_CGWJ, stop_rule=STOP_REFERENCE, eps=EPS_REF, max_it=0, check=True):
        it = C.c_long()
        rv = _lib.load().ufem_solve(self.h, solver, stop_rule, eps, max_it, C.byref(it))
        if check:
            _lib.check("ufem_solve", rv)
        return rv, it.value

    def fem_solve(self, solver=SOLVER_CGWJ, check=True):
        it = C.c_long()
        rv = _lib.load().ufem_fem_solve(self.h, solver, C.byref(it))
        if check:
            _lib.check("ufem_fem_solve", rv)
        return rv, it.value

    # ---- results -----------------------------------------------------------------
    def u(self) -> np.ndarray:
        out = np.zeros(self.ndof)
        _lib.check("ufem_get_u", _lib.load().ufem_get_u(self.h, _dp(out)))
        return out

    def set_u(self, u):
        u = np.ascontiguousarray(u, np.float64)
        _lib.check("ufem_set_u", _lib.load().ufem_set_u(self.h, _dp(u)))

    def F(self) -> np.ndarray:
        out = np.zeros(self.ndof)
        _lib.check("ufem_get_F", _lib.load().ufem_get_F(self.h, _dp(out)))
        return out

    def K_values(self) -> np.ndarray:
        b, nbr, nnzb = self.bsr_shape()
        out = np.zeros(nnzb * b * b)
        _lib.check("ufem_get_K_values", _lib.load().ufem_get_K_values(self.h, _dp(out)))
        return out.reshape(nnzb, b, b)

    def element_matrices(self, e_len: int, size: int) -> np.ndarray:
        out = np.zeros(e_len * size * size)
        _lib.check("ufem_get_element_matrices", _lib.load().ufem_get_element_matrices(self.h, _dp(out)))
        return out.reshape(e_len, size, size)

    def stresses(self, e_len: int, quad: bool):
        nip, ns = (4, 3) if quad else (27, 6)
        sig = np.zeros(e_len * nip * ns)
        vm = np.zeros(e_len * nip)
        _lib.check("ufem_get_stresses", _lib.load().ufem_get_stresses(self.h, _dp(sig), _dp(vm)))
        return sig.reshape(e_len, nip, ns), vm.reshape(e_len, nip)

    def reactions(self):
        L = _lib.load()
        n = L.ufem_num_reactions(self.h)
        node, dof, val = np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n)
        _lib.check("ufem_get_reactions", L.ufem_get_reactions(self.h, _lp(node), _lp(dof), _dp(val)))
        return node, dof, val

    def ingest_ms(self):
        v = np.zeros(6)
        _lib.check("ufem_get_ingest_ms", _lib.load().ufem_get_ingest_ms(self.h, _dp(v)))
        return dict(zip(("read", "parse", "tables", "pattern", "loads", "upload"), v.tolist()))

    def phase_ms(self):
        v = [C.c_double() for _ in range(4)]
        _lib.load().ufem_get_phase_ms(self.h, *[C.byref(x) for x in v])
        return dict(fill=v[0].value, bcs=v[1].value, solve=v[2].value, results=v[3].value)


def bsr_to_dense(rp, ci, vals, b):
    """Dense matrix from the block-sparse pattern and values (tests only, small)."""
    nbr = len(rp) - 1
    A = np.zeros((nbr * b, nbr * b))
    for I in range(nbr):
        for k in range(rp[I], rp[I + 1]):
            J = ci[k]
            A[I * b:(I + 1) * b, J * b:(J + 1) * b] = vals[k]
    return A


def rowslot_to_dense(fp, dp, pos, data):
    n = len(fp)
    A = np.zeros((n, n))
    for i in range(n):
        for j in range(fp[i], fp[i] + dp[i]):
            if pos[j] <= 0:
                break
            A[i, pos[j] - 1] = data[j]
    return A


def eqs(which: str, fp, dp, pos, data, b, x0, eps=EPS_REF, max_it=None):
    """The level-1 drop-in: femEqsCGwJ / femEqsBiCCSwJ / femEqsCGwSSOR on the
    reference's row-slot matrix, solved on the GPU."""
    L = _lib.load()
    fn = {"cgwj": L.ufem_eqs_cgwj, "bicg": L.ufem_eqs_bicgs, "ssor": L.ufem_eqs_cgwssor}[which]
    fp = np.ascontiguousarray(fp, np.int64)
    dp = np.ascontiguousarray(dp, np.int64)
    pos = np.ascontiguousarray(pos, np.int64)
    data = np.ascontiguousarray(data, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.array(x0, dtype=np.float64, copy=True)
    rv = fn(len(fp), _lp(fp), _lp(dp), _lp(pos), _dp(data), _dp(b), _dp(x), eps,
            len(fp) if max_it is None else max_it)
    return rv, x
