"""The BF16 tensor-core MLP of the learned initial guess against a numpy
restatement that rounds every matrix-product operand to BF16 the way the
kernel does (round to nearest even) and accumulates in float64.

Tolerances: forward outputs 2e-3, parameter gradients 2e-2 relative to the
largest entry (the kernel accumulates in FP32 and evaluates tanh in FP32)."""
import numpy as np
import pytest

from nrpyelliptic_b200 import _lib

pytestmark = pytest.mark.gpu


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def mm(a, b):
    return bf16(a) @ bf16(b)


def unpack(p, dims):
    out, o = [], 0
    for i in range(len(dims) - 1):
        n_w = dims[i] * dims[i + 1]
        W = p[o:o + n_w].reshape(dims[i], dims[i + 1]).astype(np.float64)
        o += n_w
        b = p[o:o + dims[i + 1]].astype(np.float64)
        o += dims[i + 1]
        out.append((W, b))
    return out


def forward(layers, x):
    hs = [x.astype(np.float64)]
    for i, (W, b) in enumerate(layers):
        z = mm(hs[-1], W) + b
        hs.append(np.tanh(z) if i + 1 < len(layers) else z)
    return hs


def grads(layers, x, t):
    hs = forward(layers, x)
    y = hs[-1]
    dz = 2.0 * (y - t) / y.size
    g = []
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        g.append((mm(hs[i].T, dz), dz.sum(0)))
        if i > 0:
            dz = mm(dz, W.T) * (1.0 - hs[i] ** 2)
    return ((y - t) ** 2).mean(), g[::-1]


class Dev:
    """Device FP32 copy of an array."""

    def __init__(self, lib, a):
        self.lib, self.a = lib, np.ascontiguousarray(a, dtype=np.float32)
        self.p = lib.nrpyell_device_malloc(self.a.nbytes)
        lib.nrpyell_memcpy(self.p, self.a.ctypes.data, self.a.nbytes, 0)

    def get(self, shape):
        out = np.empty(shape, np.float32)
        self.lib.nrpyell_memcpy(out.ctypes.data, self.p, out.nbytes, 1)
        return out

    def free(self):
        self.lib.nrpyell_device_free(self.p)


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    return lib


def test_forward_and_gradient_match_bf16_restatement(lib):
    dims = [13, 96, 96, 40]
    m = lib.nrpyell_mlp_create(13, 96, 2, 40, 128, 7)
    _lib.check(lib)
    rng = np.random.default_rng(3)
    x = rng.normal(size=(77, 13)).astype(np.float32)
    t = rng.normal(size=(77, 40)).astype(np.float32)
    p = np.empty(lib.nrpyell_mlp_num_params(m), np.float32)
    lib.nrpyell_mlp_get_params(m, p.ctypes.data)
    layers = unpack(p, dims)
    dx, dt_ = Dev(lib, x), Dev(lib, t)
    dy = Dev(lib, np.zeros((77, 40)))
    assert lib.nrpyell_mlp_predict(m, dx.p, 77, dy.p) == 0
    y = dy.get((77, 40))
    y_ref = forward(layers, x)[-1]
    assert np.max(np.abs(y - y_ref)) < 2e-3 * np.max(np.abs(y_ref))
    g = np.empty_like(p)
    loss = lib.nrpyell_mlp_loss_grad(m, dx.p, dt_.p, 77, g.ctypes.data)
    loss_ref, g_ref = grads(layers, x, t)
    assert abs(loss - loss_ref) < 1e-3 * loss_ref
    for (gW, gb), (rW, rb) in zip(unpack(g, dims), g_ref):
        assert np.max(np.abs(gW - rW)) < 2e-2 * np.max(np.abs(rW))
        assert np.max(np.abs(gb - rb)) < 2e-2 * np.max(np.abs(rb))
    for d in (dx, dt_, dy):
        d.free()
    lib.nrpyell_mlp_destroy(m)


def test_training_fits_a_smooth_map(lib):
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(2048, 13)).astype(np.float32)
    A = rng.normal(size=(13, 32)) / 4
    t = np.sin(x @ A).astype(np.float32)
    m = lib.nrpyell_mlp_create(13, 128, 3, 32, 256, 11)
    dx, dt_ = Dev(lib, x), Dev(lib, t)
    hist = np.zeros(60)
    last = lib.nrpyell_mlp_train(m, dx.p, dt_.p, 2048, 256, 60, 2e-3, 1, hist.ctypes.data)
    _lib.check(lib)
    assert last == hist[-1] and hist[0] > 0 and 0 < last < 0.05 * hist[0], hist[[0, 10, 30, 59]]
    # predictions after training reproduce the reported loss
    dy = Dev(lib, np.zeros((2048, 32)))
    lib.nrpyell_mlp_predict(m, dx.p, 2048, dy.p)
    mse = float(np.mean((dy.get((2048, 32)) - t) ** 2))
    assert mse < 2 * last
    for d in (dx, dt_, dy):
        d.free()
    lib.nrpyell_mlp_destroy(m)
