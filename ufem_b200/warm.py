"""Learned warm start of the batched Monte Carlo solve (``ufem_warm_*``).

No counterpart in the reference: its only hook is the disabled warm start of
monte_linear_solver (fem/fem_mont.c:493-504).  Training solves samples with
the batched GPU solver, builds a POD basis of their solutions and trains the
tensor-core MLP to predict POD coefficients from the samples' inputs; the
warm-started solve uses the prediction as the PCG initial guess and still
iterates to the same tolerance, falling back to a solve from zero for any
sample whose iterations regress.  Device memory comes from torch (plumbing
only); every computation runs in libufem_gpu.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .api import GpuModel
from .mc import default_options


def default_warm_options():
    o = _lib.WarmOptions()
    _lib.load().ufem_warm_default_options(C.byref(o))
    return o


def _dev(a, dtype):
    import torch
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype).contiguous()


def _fields(s) -> dict:
    out = {}
    for f, _ in s._fields_:
        v = getattr(s, f)
        out[f] = list(v) if hasattr(v, "__len__") else v
    return out


class WarmStart:
    """POD basis + MLP warm start for one model (``ufem_warm`` handle)."""

    def __init__(self, model: GpuModel, feat_cols, feat_log=None, scale_col: int = -1, **opts):
        self.L = _lib.load()
        self.model = model
        o = default_warm_options()
        o.n_feat = len(feat_cols)
        for i, c in enumerate(feat_cols):
            o.feat_cols[i] = int(c)
            o.feat_log[i] = int(feat_log[i]) if feat_log is not None else 0
        o.scale_col = int(scale_col)
        for k, v in opts.items():
            setattr(o, k, v)
        self.opts = o
        h = C.c_void_p()
        _lib.check("ufem_warm_create", self.L.ufem_warm_create(model.h, C.byref(o), C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.ufem_warm_free(self.h)
            self.h = None

    @staticmethod
    def _mc_opts(precision, tol, coarse=True):
        opt = default_options()
        opt.precision = precision
        opt.tol = tol
        opt.coarse = int(bool(coarse))
        return opt

    def train(self, ifld, precision: int = 1, tol: float = 1e-8) -> dict:
        import torch
        d = _dev(ifld, torch.float64)
        st = _lib.WarmTrainStats()
        opt = self._mc_opts(precision, tol)
        _lib.check("ufem_warm_train", self.L.ufem_warm_train(self.h, d.shape[0], d.data_ptr(), C.byref(opt),
                                                             C.byref(st)))
        return _fields(st)

    def guess(self, ifld) -> np.ndarray:
        import torch
        d = _dev(ifld, torch.float64)
        out = torch.empty((d.shape[0], self.model.ndof), dtype=torch.float64, device="cuda")
        _lib.check("ufem_warm_guess", self.L.ufem_warm_guess(self.h, d.shape[0], d.data_ptr(), out.data_ptr()))
        return out.cpu().numpy()

    def set_guess_mode(self, mode: int) -> None:
        """0: the MLP's coefficients; 1: each sample's POD-Galerkin coefficients."""
        _lib.check("ufem_warm_set_guess_mode", self.L.ufem_warm_set_guess_mode(self.h, int(mode)))

    def set_guess_scale(self, factor: float) -> None:
        _lib.check("ufem_warm_set_guess_scale", self.L.ufem_warm_set_guess_scale(self.h, float(factor)))

    def solve(self, ifld, precision: int = 1, tol: float = 1e-8, coarse: bool = True, tiles_per_block: int = 0):
        """Warm-started batched solve: (ofld, status, iters, stats).  With
        ``coarse`` (precision 2) the preconditioner adds the coarse correction
        on the leading POD modes that training set on the model;
        ``tiles_per_block`` > 0 overrides the launch shape's work tiles per
        persistent block."""
        import torch
        d = _dev(ifld, torch.float64)
        n = d.shape[0]
        olen = max(1, self.model.model.mc_olen)
        of = torch.zeros((n, olen), dtype=torch.float64, device="cuda")
        st = torch.zeros(n, dtype=torch.int32, device="cuda")
        it = torch.zeros(n, dtype=torch.int64, device="cuda")
        ws = _lib.WarmStats()
        opt = self._mc_opts(precision, tol, coarse)
        opt.tiles_per_block = int(tiles_per_block)
        _lib.check("ufem_warm_solve", self.L.ufem_warm_solve(self.h, n, d.data_ptr(), of.data_ptr(), st.data_ptr(),
                                                             it.data_ptr(), C.byref(opt), C.byref(ws)))
        return (of.cpu().numpy()[:, :self.model.model.mc_olen], st.cpu().numpy(), it.cpu().numpy(), _fields(ws))

    def basis(self):
        r = self.opts.n_modes
        phi = np.zeros((self.model.ndof, r))
        s2 = np.zeros(r)
        _lib.check("ufem_warm_get_basis", self.L.ufem_warm_get_basis(
            self.h, phi.ctypes.data_as(C.POINTER(C.c_double)), s2.ctypes.data_as(C.POINTER(C.c_double))))
        return phi, s2
