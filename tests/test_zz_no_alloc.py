"""The allocation-free Jacobi PCG (ufem_eqs_cgwj_noalloc).

It is meant for callers that may not allocate device memory while they
solve (an application whose allocator owns the device pool, a solve issued
from another GPU library's callback, a loop that must not hit cudaMalloc's
implicit synchronisation).  Its scratch lives in one array built into the
library, so it takes the matrix and vectors already in device memory.

The test solves the same supported beam system through the new entry point
and through the existing ufem_eqs_cgwj (which uploads the reference's
row-slot matrix itself), twice in a row, and compares the solutions within
the 1e-8 relative tolerance of the other displacement tests.  It also checks
that the second call changes no device memory reservation and that an
oversized system is refused.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U_TOL = 1e-8


def _system():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    m = mg.beam_brick(20, 5, 5, 8.0, 2.0, 2.0)
    g = GpuModel(m)
    g.fill_K(0)
    g.add_loads()
    g.add_disps()
    b, nbr, nnzb = g.bsr_shape()
    rp, ci = g.bsr_pattern()
    vals = g.K_values()
    F = g.F()
    return g, b, nbr, rp, ci, vals, F


def _to_rowslot(b, nbr, rp, ci, vals):
    """The same matrix in the reference's row-slot layout (1-based columns)."""
    n = nbr * b
    frompos, defpos, pos, data = [], [], [], []
    off = 0
    for I in range(nbr):
        for a in range(b):
            cols = []
            for k in range(rp[I], rp[I + 1]):
                for c in range(b):
                    cols.append((ci[k] * b + c + 1, vals[k, a, c]))
            frompos.append(off)
            defpos.append(len(cols))
            for col, v in cols:
                pos.append(col)
                data.append(v)
            off += len(cols)
    return (np.array(frompos, np.int64), np.array(defpos, np.int64), np.array(pos, np.int64),
            np.array(data, np.float64))


def test_noalloc_matches_existing_entry_point_twice():
    import torch
    from ufem_b200 import _lib, api
    L = _lib.load()
    g, b, nbr, rp, ci, vals, F = _system()
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(rp.astype(np.int32)).to(dev)
    d_ci = torch.from_numpy(ci.astype(np.int32)).to(dev)
    d_val = torch.from_numpy(np.ascontiguousarray(vals.reshape(-1))).to(dev)
    d_b = torch.from_numpy(F).to(dev)
    # the existing entry point on the reference's own matrix layout
    fp, dp, pos, data = _to_rowslot(b, nbr, rp, ci, vals)
    rv, x_ref = api.eqs("cgwj", fp, dp, pos, data, F, np.zeros(len(F)))
    assert rv == 0
    sols = []
    free_after = []
    for call in range(2):
        d_x = torch.zeros(len(F), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        it = C.c_long()
        rv = L.ufem_eqs_cgwj_noalloc(b, nbr, d_rp.data_ptr(), d_ci.data_ptr(), d_val.data_ptr(), d_b.data_ptr(),
                                     d_x.data_ptr(), api.EPS_REF, len(F), C.byref(it))
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info(0)[0])
        assert rv == 0, L.ufem_last_error()
        assert it.value > 0
        x = d_x.cpu().numpy()
        err = np.abs(x - x_ref).max() / np.abs(x_ref).max()
        assert err <= U_TOL, (call, err)
        sols.append(x)
    # the shared scratch keeps the previous call's contents; the second call
    # must not depend on them
    assert np.abs(sols[0] - sols[1]).max() <= U_TOL * np.abs(sols[0]).max()
    # nothing was reserved on the device by the second call
    assert free_after[0] == free_after[1]


def test_noalloc_refuses_oversized_systems():
    from ufem_b200 import _lib, api
    L = _lib.load()
    it = C.c_long()
    rv = L.ufem_eqs_cgwj_noalloc(3, 131072, None, None, None, None, None, api.EPS_REF, 10, C.byref(it))
    assert rv == -9                              # AF_ERR_SIZ
    assert b"131072" in L.ufem_last_error()
