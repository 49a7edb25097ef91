"""Monte Carlo on the GPU: the reference's plugin ABI and the batched solve.

``MonteLib`` calls the ``monte_*`` functions of libufem_gpu.so exactly as an
external driver calls libfem.so's (fem/fem_mont.c:137-866).  ``mc_solve``
runs many samples of several meshes in one batched launch
(``ufem_mc_solve``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .api import GpuModel, _dp, _ip, _lp

ST_CONVERGED, ST_MAXIT, ST_BREAKDOWN, ST_NAN, ST_FALLBACK = 0, 1, 2, 3, 4


class MonteLib:
    """The libfem.so plugin interface (interface type 2) on the GPU."""

    def __init__(self, param: str):
        self.L = _lib.load()
        self.param = param.encode()
        rv = self.L.monte_init_lib_stuff(self.param)
        if rv != 0:
            raise _lib.UfemError("monte_init_lib_stuff", rv)
        il, ol, ff = C.c_long(), C.c_long(), C.c_long()
        self.L.monte_nums_of_vars(self.param, C.byref(il), C.byref(ol), C.byref(ff))
        self.ilen, self.olen, self.ffunc = il.value, ol.value, ff.value

    def interface_type(self) -> int:
        return self.L.monte_dlib_interface_type()

    def ivar_names(self):
        return [self.L.monte_ivar_name(self.param, i).decode() for i in range(self.ilen)]

    def ovar_names(self):
        return [self.L.monte_ovar_name(self.param, i).decode() for i in range(self.olen)]

    def solution(self, ifld: np.ndarray, if_type: int = 0) -> tuple[int, np.ndarray]:
        ifld = np.ascontiguousarray(ifld, np.float64)
        ofld = np.zeros(max(self.olen, 1))
        rv = self.L.monte_solution(self.param, _dp(ifld), _dp(ofld), if_type)
        return rv, ofld[:self.olen]

    def solution_batch(self, ifld: np.ndarray, if_type: int = 0):
        ifld = np.ascontiguousarray(ifld, np.float64)
        n = ifld.shape[0]
        ofld = np.zeros((n, max(self.olen, 1)))
        status = np.zeros(n, np.int32)
        rv = self.L.monte_solution_batch(self.param, n, _dp(ifld), _dp(ofld), if_type, _ip(status))
        return rv, ofld[:, :self.olen], status

    def close(self):
        self.L.monte_clean_lib_stuff(self.param)


def default_options():
    o = _lib.McOptions()
    _lib.load().ufem_mc_default_options(C.byref(o))
    return o


def mc_solve(models: list[GpuModel], iflds: list[np.ndarray], precision: int = 1, tol: float = 1e-8,
             max_iters: int | None = None, replace_every: int | None = None, replace_near: float | None = None,
             u_guess: list[np.ndarray | None] | None = None, olens: list[int] | None = None,
             tiles_per_block: int = 0, unroll: int = 0, lane_samples: int = 0, coarse: int = 1):
    """Batched solve of every sample of every mesh in one launch.

    Returns per mesh (ofld[nsamp, olen], status[nsamp], iters[nsamp]) and the
    launch statistics."""
    L = _lib.load()
    nm = len(models)
    opt = default_options()
    opt.precision = precision
    opt.tol = tol
    if max_iters is not None:
        opt.max_iters = max_iters
    if replace_every is not None:
        opt.replace_every = replace_every
    if replace_near is not None:
        opt.replace_near = replace_near
    opt.tiles_per_block = tiles_per_block
    opt.unroll = unroll
    opt.lane_samples = lane_samples
    opt.coarse = coarse
    keep = []
    hs = (C.c_void_p * nm)(*[m.h.value for m in models])
    ns = np.array([f.shape[0] for f in iflds], np.int64)
    pin = (C.POINTER(C.c_double) * nm)()
    pout = (C.POINTER(C.c_double) * nm)()
    pst = (C.POINTER(C.c_int) * nm)()
    pit = (C.POINTER(C.c_long) * nm)()
    pg = (C.POINTER(C.c_double) * nm)()
    outs = []
    for k in range(nm):
        f = np.ascontiguousarray(iflds[k], np.float64)
        olen = olens[k] if olens else models[k].model.mc_olen
        o = np.zeros((f.shape[0], max(olen, 1)))
        st = np.zeros(f.shape[0], np.int32)
        it = np.zeros(f.shape[0], np.int64)
        keep += [f, o, st, it]
        pin[k], pout[k], pst[k], pit[k] = _dp(f), _dp(o), _ip(st), _lp(it)
        if u_guess is not None and u_guess[k] is not None:
            g = np.ascontiguousarray(u_guess[k], np.float64)
            keep.append(g)
            pg[k] = _dp(g)
        else:
            pg[k] = C.POINTER(C.c_double)()
        outs.append((o, st, it, olen))
    rv = L.ufem_mc_solve(nm, hs, _lp(ns), pin, pout, pst, pit, pg, C.byref(opt))
    _lib.check("ufem_mc_solve", rv)
    stats = _lib.McStats()
    L.ufem_mc_get_stats(C.byref(stats))
    res = [(o[:, :olen], st, it) for (o, st, it, olen) in outs]
    return res, stats


def set_coarse(model: GpuModel, Wc) -> None:
    """Coarse space of the preconditioner of ``model``'s precision-2 solves,
    M^-1 = D^-1 + Wc Wc^T (``ufem_mc_set_coarse``); ``Wc`` [nDOFAct x m]
    (m a multiple of 16, at most 128), or None to remove it."""
    import torch
    L = _lib.load()
    if Wc is None:
        _lib.check("ufem_mc_set_coarse", L.ufem_mc_set_coarse(model.h, 0, None))
        return
    d = torch.as_tensor(np.ascontiguousarray(Wc, np.float64)).cuda()
    _lib.check("ufem_mc_set_coarse", L.ufem_mc_set_coarse(model.h, int(d.shape[1]), C.c_void_p(d.data_ptr())))
    torch.cuda.synchronize()


def stats_dict(s) -> dict:
    return {f: getattr(s, f) for f, _ in s._fields_}


def mc_solve_serial(model: GpuModel, ifld: np.ndarray, tol: float = 1e-8):
    """The plain method: one sample at a time, FP64 assembly + FP64 Jacobi PCG."""
    L = _lib.load()
    f = np.ascontiguousarray(ifld, np.float64)
    n = f.shape[0]
    olen = model.model.mc_olen
    o = np.zeros((n, max(olen, 1)))
    st = np.zeros(n, np.int32)
    it = np.zeros(n, np.int64)
    _lib.check("ufem_mc_solve_serial", L.ufem_mc_solve_serial(model.h, n, _dp(f), _dp(o), _ip(st), _lp(it), tol))
    return o[:, :olen], st, it


def autotune(models: list[GpuModel], iflds, precision: int = 2, tol: float = 1e-8, cache_path: str | None = None):
    """Pick the batched solve's launch shape for this batch (``ufem_mc_autotune``)
    and return the tuned options; later solves of batches of the same shape
    pick it up from the cache by themselves."""
    import torch
    L = _lib.load()
    nm = len(models)
    d = [f if isinstance(f, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(f, np.float64)).cuda()
         for f in iflds]
    ns = np.array([t.shape[0] for t in d], np.int64)
    opt = default_options()
    opt.precision = precision
    opt.tol = tol
    best = _lib.McOptions()
    rv = L.ufem_mc_autotune(nm, (C.c_void_p * nm)(*[m.h.value for m in models]), _lp(ns),
                            (C.c_void_p * nm)(*[t.data_ptr() for t in d]), C.byref(opt),
                            cache_path.encode() if cache_path else None, C.byref(best))
    _lib.check("ufem_mc_autotune", rv)
    return best
