"""The learned planner's network: BF16/FP32 kernels checked against an FP64 CPU model.

The reference has no learned component; the check is the standard one for a
training kernel: forward outputs and every parameter gradient of the masked MSE
loss agree with a NumPy FP64 implementation of the same network evaluated on the
same BF16-rounded operands, within the tolerance BF16 operands allow.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 3e-2  # relative (to the largest magnitude of each tensor): BF16 operands, FP32 accumulation


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p, nin, nh, nout):
    at = 0
    out = []
    for shape in [(nin, nh), (nh,), (nh, nh), (nh,), (nh, nout), (nout,)]:
        n = int(np.prod(shape))
        out.append(p[at:at + n].reshape(shape).astype(np.float64))
        at += n
    return out


def cpu_model(params, x, t, mask, nin, nh, nout):
    W1, b1, W2, b2, W3, b3 = unpack(params, nin, nh, nout)
    x = x.astype(np.float64)
    h1 = np.maximum(bf16(x) @ bf16(W1) + b1, 0)
    h2 = np.maximum(bf16(h1) @ bf16(W2) + b2, 0)
    y = bf16(h2) @ bf16(W3) + b3
    norm = max(1.0, mask.sum())
    d = (y - t) * mask
    loss = (d * d).sum() / norm
    dy = 2 * d / norm
    gW3 = bf16(h2).T @ bf16(dy)
    gb3 = dy.sum(0)
    dh2 = (bf16(dy) @ bf16(W3).T) * (h2 > 0)
    gW2 = bf16(h1).T @ bf16(dh2)
    gb2 = dh2.sum(0)
    dh1 = (bf16(dh2) @ bf16(W2).T) * (h1 > 0)
    gW1 = bf16(x).T @ bf16(dh1)
    gb1 = dh1.sum(0)
    return y, loss, [gW1, gb1, gW2, gb2, gW3, gb3]


def close(a, b):
    scale = max(np.abs(b).max(), 1e-6)
    return np.abs(a - b).max() / scale


@pytest.fixture(scope="module")
def mlp(vs):
    L = vs.capi.lib()
    h = C.c_void_p()
    nin, nh, nout = 76, 128, 720
    vs.capi.check(L.vsgm_mlp_create(0, nin, nh, nout, 7, C.byref(h)))
    yield L, h, nin, nh, nout
    L.vsgm_mlp_destroy(h)


def test_forward_and_gradients_match_fp64(vs, mlp):
    L, h, nin, nh, nout = mlp
    rng = np.random.default_rng(1)
    B = 96  # not a multiple of the 64-row tile: exercises the edges
    x = rng.normal(size=(B, nin)).astype(np.float32)
    t = rng.normal(size=(B, nout)).astype(np.float32)
    mask = (rng.random((B, nout)) < 0.05).astype(np.float32)
    n = L.vsgm_mlp_num_params(h)
    params = np.zeros(n, np.float32)
    vs.capi.check(L.vsgm_mlp_get_params(h, params.ctypes.data_as(C.POINTER(C.c_float))))
    y = np.zeros((B, nout), np.float32)
    L.vsgm_mlp_forward(h, x.ctypes.data_as(C.POINTER(C.c_float)), B, y.ctypes.data_as(C.POINTER(C.c_float)))
    loss = C.c_float()
    grads = np.zeros(n, np.float32)
    vs.capi.check(L.vsgm_mlp_gradients(h, x.ctypes.data_as(C.POINTER(C.c_float)), t.ctypes.data_as(C.POINTER(C.c_float)),
                                       mask.ctypes.data_as(C.POINTER(C.c_float)), B, C.byref(loss),
                                       grads.ctypes.data_as(C.POINTER(C.c_float))))
    y_ref, loss_ref, g_ref = cpu_model(params, x, t, mask, nin, nh, nout)
    assert close(y, y_ref) < TOL
    assert abs(loss.value - loss_ref) / loss_ref < TOL
    for got, want in zip(unpack(grads, nin, nh, nout), g_ref):
        assert close(got, want) < TOL


def test_training_reduces_loss(vs, mlp):
    L, h, nin, nh, nout = mlp
    rng = np.random.default_rng(2)
    B = 256
    x = rng.normal(size=(B, nin)).astype(np.float32)
    Wt = rng.normal(size=(nin, nout)).astype(np.float32) / np.sqrt(nin)
    t = (x @ Wt).astype(np.float32)
    mask = (rng.random((B, nout)) < 0.1).astype(np.float32)
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    loss = C.c_float()
    first = None
    for step in range(300):
        vs.capi.check(L.vsgm_mlp_train_step(h, P(x), P(t), P(mask), B, 3e-3, C.byref(loss)))
        if first is None:
            first = loss.value
    assert loss.value < 0.2 * first
