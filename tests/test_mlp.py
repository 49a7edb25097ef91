"""The warm-start MLP: its CPU oracle (finite differences), the tensor-core
GEMM against numpy, the GPU gradients against the oracle, and training.

Tolerances: the GEMM takes BF16 operands and accumulates in FP32, so it is
compared with the FP64 product of the same BF16 values at 1e-5 relative;
the GPU gradients are compared with the oracle evaluated with the same BF16
rounding points at 2e-2 relative per parameter tensor (FP32 accumulation
order and erf/exp implementations differ)."""
import ctypes as C

import numpy as np
import pytest

from oracle import mlp_oracle as mo

H, NOUT, NIN = 64, 32, 17


def _params(seed=0):
    rng = np.random.default_rng(seed)
    W1 = np.zeros((H, mo.N_INP))
    W1[:, :NIN] = rng.uniform(-0.5, 0.5, (H, NIN))
    return np.concatenate([W1.ravel(), rng.normal(0, 0.1, H), rng.uniform(-0.2, 0.2, H * H),
                           rng.normal(0, 0.1, H), rng.uniform(-0.2, 0.2, NOUT * H), rng.normal(0, 0.1, NOUT)])


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    X = rng.normal(size=(8, NIN))
    T = rng.normal(size=(8, NOUT))
    p = _params()
    _, g = mo.loss_and_grads(p, X, T, H, NOUT, bf=False)
    W1mask = np.zeros_like(p, bool)
    W1mask[:H * mo.N_INP] = (np.arange(H * mo.N_INP) % mo.N_INP) >= NIN   # padded inputs
    idx = rng.choice(np.nonzero(~W1mask)[0], 40, replace=False)
    for i in idx:
        e = np.zeros_like(p)
        h = 1e-6 * max(1.0, abs(p[i]))
        e[i] = h
        lp, _ = mo.loss_and_grads(p + e, X, T, H, NOUT, bf=False)
        lm, _ = mo.loss_and_grads(p - e, X, T, H, NOUT, bf=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])) + 1e-9, (i, fd, g[i])


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 64, 256), (64, 32, 4096), (256, 256, 520)])
def test_tensor_core_gemm(M, N, K):
    import torch
    from ufem_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(M + N + K)
    A = mo.bf16(rng.normal(size=(M, K)))
    B = mo.bf16(rng.normal(size=(N, K)))
    dA = torch.tensor(A, dtype=torch.bfloat16, device="cuda")
    dB = torch.tensor(B, dtype=torch.bfloat16, device="cuda")
    dC = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    rv = L.ufem_tc_gemm_bf16(M, N, K, dA.data_ptr(), dB.data_ptr(), dC.data_ptr())
    assert rv == 0, L.ufem_last_error()
    ref = A @ B.T
    err = np.abs(dC.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err <= 1e-5, err


def _gpu_mlp(params):
    from ufem_b200 import _lib
    L = _lib.load()
    h = C.c_void_p()
    assert L.ufem_mlp_create(NIN, H, NOUT, 7, C.byref(h)) == 0
    assert L.ufem_mlp_num_params(h) == len(params)
    p32 = np.ascontiguousarray(params, np.float32)
    assert L.ufem_mlp_set_params(h, p32.ctypes.data_as(C.POINTER(C.c_float))) == 0
    return L, h


@pytest.mark.gpu
def test_gpu_gradients_match_oracle():
    import torch
    rng = np.random.default_rng(3)
    B = 300
    X = rng.normal(size=(B, NIN)).astype(np.float32)
    T = rng.normal(size=(B, NOUT)).astype(np.float32)
    p = _params(5).astype(np.float32).astype(np.float64)
    L, h = _gpu_mlp(p)
    dX = torch.tensor(X, device="cuda")
    dT = torch.tensor(T, device="cuda")
    g = np.zeros(len(p), np.float32)
    loss = C.c_float()
    rv = L.ufem_mlp_gradients(h, B, dX.data_ptr(), dT.data_ptr(), g.ctypes.data_as(C.POINTER(C.c_float)),
                              C.byref(loss))
    assert rv == 0, L.ufem_last_error()
    lref, gref = mo.loss_and_grads(p, X.astype(np.float64), T.astype(np.float64), H, NOUT, bf=True)
    assert abs(loss.value - lref) <= 1e-3 * lref
    sizes = [H * mo.N_INP, H, H * H, H, NOUT * H, NOUT]
    o = 0
    for s in sizes:
        a, b = g[o:o + s].astype(np.float64), gref[o:o + s]
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b), (o, np.linalg.norm(a - b) / np.linalg.norm(b))
        o += s
    # forward outputs against the oracle
    y = torch.zeros((B, NOUT), device="cuda")
    assert L.ufem_mlp_forward(h, B, dX.data_ptr(), y.data_ptr()) == 0
    yref = mo.forward(p, X.astype(np.float64), H, NOUT, bf=True)["Y"]
    assert np.abs(y.cpu().numpy() - yref).max() <= 1e-3 * np.abs(yref).max()
    L.ufem_mlp_free(h)


@pytest.mark.gpu
def test_gpu_training_reduces_loss():
    import torch
    from ufem_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(4)
    B = 512
    X = rng.normal(size=(B, NIN)).astype(np.float32)
    Wt = rng.normal(size=(NIN, NOUT)) / np.sqrt(NIN)
    T = np.tanh(X @ Wt).astype(np.float32)
    h = C.c_void_p()
    assert L.ufem_mlp_create(NIN, H, NOUT, 11, C.byref(h)) == 0
    dX, dT = torch.tensor(X, device="cuda"), torch.tensor(T, device="cuda")
    loss = C.c_float()
    losses = []
    for it in range(300):
        rv = L.ufem_mlp_train_step(h, B, dX.data_ptr(), dT.data_ptr(), 3e-3, C.byref(loss))
        assert rv == 0, L.ufem_last_error()
        losses.append(loss.value)
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])
    L.ufem_mlp_free(h)
