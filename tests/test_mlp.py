"""The warm-start network: the CPU oracle (oracle/mlp_oracle.py) against finite differences, the
library's layout and argument checks (CPU), and the tcgen05 kernels against the oracle (GPU).

Tolerances: the GPU and the oracle round to bfloat16 at the same places but accumulate in a different
order (fp32 tensor-core sums against float64), so an element can land one bf16 step apart; outputs
are held to 1e-2 absolute + 1e-2 relative, gradients to 2e-2 in relative norm per layer, the loss to
1e-3 relative, one Adam step to 1e-5 relative (plus the float32 rounding of m and v).
"""
import ctypes as C

import numpy as np
import pytest

import mlp_oracle as MO
from bmc_b200 import _lib

SMALL = (10, 128, 2, 3)          # n_in, n_hidden, hidden layers, n_out
LADDER = (244, 256, 3, 6)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 1e-3], np.float32)
    r = MO.bf16(x)
    assert r[0] == 1.0 and r[3] == -2.5 and r[4] == 0.0
    assert r[1] == 1.0                                   # halfway, ties to the even neighbour
    assert r[2] == np.float32(1.0 + 2 ** -7)              # above halfway rounds up
    assert abs(r[5] / 1e-3 - 1) < 2 ** -8


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = MO.init_params(*SMALL, seed=1).astype(np.float64)
    x = rng.normal(size=(7, SMALL[0]))
    t = rng.normal(size=(7, SMALL[3]))
    y, cache = MO.forward(p, SMALL, x, emulate=False)
    g, loss = MO.backward(p, SMALL, cache, t)
    lay = MO.layout(*SMALL)
    real = [(l, i) for l in lay for i in range(l.off_w, l.off_b + l.rows) if g[i] != 0.0]
    pick = rng.choice(len(real), 40, replace=False)
    for j in pick:
        i = real[j][1]
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = MO.backward(pp, SMALL, MO.forward(pp, SMALL, x, emulate=False)[1], t)[1]
        lm = MO.backward(pm, SMALL, MO.forward(pm, SMALL, x, emulate=False)[1], t)[1]
        assert g[i] == pytest.approx((lp - lm) / (2 * h), rel=1e-5, abs=1e-9)
    # padded weights have zero gradient
    L0 = lay[0]
    W0 = g[L0.off_w:L0.off_b].reshape(L0.rows, L0.cols)
    assert not W0[:, SMALL[0]:].any()


def test_oracle_adam_is_bias_corrected():
    p, g = np.ones(3), np.array([0.5, -1.0, 0.0])
    p1, m, v = MO.adam(p, g, np.zeros(3), np.zeros(3), 1, lr=1e-3)
    # the first corrected step moves each weight by lr * sign(g)
    np.testing.assert_allclose(p1, [1 - 1e-3, 1 + 1e-3, 1.0], rtol=0, atol=1e-9)


def test_library_layout_and_sizes():
    from bmc_b200.warmstart import MLP
    L = _lib.lib()
    sh = _lib.MlpShape(*LADDER)
    n_p, sh_b, wb = C.c_int64(), C.c_int64(), C.c_int64()
    _lib.check(L.bmc_mlp_sizes(C.byref(sh), 4096, C.byref(n_p), C.byref(sh_b), C.byref(wb)))
    lay = MO.layout(*LADDER)
    assert n_p.value == MO.n_params(lay) == MLP.init_params(*LADDER).size
    assert sh_b.value == 2 * 2 * sum(l.rows * l.cols for l in lay)
    assert wb.value > 4096 * (256 + 3 * 256) * 2
    np.testing.assert_array_equal(MLP.init_params(*LADDER, seed=4), MO.init_params(*LADDER, seed=4))


@pytest.mark.parametrize("shape,msg", [((0, 256, 3, 6), "MLP shape"), ((244, 200, 3, 6), "multiple of 128"),
                                       ((244, 256, 9, 6), "hidden layers"), ((244, 256, 3, 200), "n_out")])
def test_bad_shapes_are_refused(shape, msg):
    L = _lib.lib()
    sh = _lib.MlpShape(*shape)
    with pytest.raises(RuntimeError, match=msg):
        _lib.check(L.bmc_mlp_sizes(C.byref(sh), 16, None, None, None))


def test_bad_calls_are_refused_before_launch():
    L = _lib.lib()
    sh = _lib.MlpShape(*LADDER)
    d = C.c_void_p(256)
    with pytest.raises(RuntimeError, match="null params"):
        _lib.check(L.bmc_mlp_forward(C.byref(sh), None, d, d, None, None, 8, None, d, 0, None))
    with pytest.raises(RuntimeError, match="256-byte"):
        _lib.check(L.bmc_mlp_forward(C.byref(sh), d, d, d, None, None, 8, None, C.c_void_p(260), 0, None))
    with pytest.raises(RuntimeError, match="MLP batch"):
        _lib.check(L.bmc_mlp_backward(C.byref(sh), d, d, 0, d, d, None, None))
    with pytest.raises(RuntimeError, match="Adam"):
        _lib.check(L.bmc_mlp_adam_step(C.byref(sh), d, d, d, d, d, 0, 1e-3, 0.9, 0.999, 1e-8, None))


# ------------------------------------------------------------------------------------------------
# GPU: the tcgen05 kernels against the oracle
# ------------------------------------------------------------------------------------------------
def _net(shape, seed=0):
    from bmc_b200.warmstart import MLP
    n_in, H, nl, n_out = shape
    return MLP(n_in, n_out, H, nl, seed=seed)


def _inputs(shape, batch, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.5, 0.3, (batch, shape[0])).astype(np.float32)
    shift = rng.normal(0.5, 0.05, shape[0]).astype(np.float32)
    scale = rng.uniform(2.0, 4.0, shape[0]).astype(np.float32)
    t = rng.normal(0.0, 0.5, (batch, shape[3])).astype(np.float32)
    return x, shift, scale, t


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,batch", [(SMALL, 300), (LADDER, 300), (LADDER, 4096)])
def test_forward_matches_the_oracle(cuda, shape, batch):
    torch = cuda
    net = _net(shape, seed=2)
    x, shift, scale, _ = _inputs(shape, batch, 5)
    net.set_input_normalisation(shift, scale)
    y = net.forward(torch.as_tensor(x).cuda()).cpu().numpy()
    want, _ = MO.forward(net.params.cpu().numpy(), shape, x, shift, scale, emulate=True)
    np.testing.assert_allclose(y, want, rtol=1e-2, atol=2e-3)
    assert net.status(batch) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("shape,batch", [(SMALL, 300), (LADDER, 4096)])
def test_backward_matches_the_oracle(cuda, shape, batch):
    torch = cuda
    net = _net(shape, seed=3)
    x, shift, scale, t = _inputs(shape, batch, 6)
    net.set_input_normalisation(shift, scale)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    net.forward(torch.as_tensor(x).cuda(), keep=True)
    net.backward(torch.as_tensor(t).cuda(), loss)
    g = net.grad.cpu().numpy().astype(np.float64)
    p = net.params.cpu().numpy()
    _, cache = MO.forward(p, shape, x, shift, scale, emulate=True)
    want, want_loss = MO.backward(p, shape, cache, t)
    assert float(loss.item()) == pytest.approx(want_loss, rel=1e-3)
    for l in MO.layout(*shape):
        assert _rel(g[l.off_w:l.off_b], want[l.off_w:l.off_b]) < 2e-2
        assert _rel(g[l.off_b:l.off_b + l.rows], want[l.off_b:l.off_b + l.rows]) < 2e-2
    lay = MO.layout(*shape)
    W0 = g[lay[0].off_w:lay[0].off_b].reshape(lay[0].rows, lay[0].cols)
    Wo = g[lay[-1].off_w:lay[-1].off_b].reshape(lay[-1].rows, lay[-1].cols)
    assert not W0[:, shape[0]:].any() and not Wo[shape[3]:].any()       # padding stays exactly zero
    assert net.status(batch) == 0


@pytest.mark.gpu
def test_adam_step_and_shadow_match_the_oracle(cuda):
    torch = cuda
    net = _net(SMALL, seed=4)
    rng = np.random.default_rng(7)
    p0 = net.params.cpu().numpy().astype(np.float64)
    g = rng.normal(0, 1e-2, p0.size) * (p0 != 0)
    m0 = rng.normal(0, 1e-3, p0.size) * (p0 != 0)
    v0 = rng.uniform(0, 1e-4, p0.size) * (p0 != 0)
    net.grad.copy_(torch.as_tensor(g, dtype=torch.float32))
    net.m.copy_(torch.as_tensor(m0, dtype=torch.float32))
    net.v.copy_(torch.as_tensor(v0, dtype=torch.float32))
    net.step = 4
    net.adam(lr=1e-3)
    p1, m1, v1 = MO.adam(p0, g.astype(np.float32).astype(np.float64), m0.astype(np.float32),
                         v0.astype(np.float32), 5, lr=1e-3)
    np.testing.assert_allclose(net.params.cpu().numpy(), p1, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(net.m.cpu().numpy(), m1, rtol=1e-5, atol=2e-9)     # fp32 cancellation
    np.testing.assert_allclose(net.v.cpu().numpy(), v1, rtol=1e-5, atol=1e-11)
    # the shadow followed: a forward pass sees the new weights
    x, shift, scale, _ = _inputs(SMALL, 256, 8)
    net.set_input_normalisation(shift, scale)
    y = net.forward(torch.as_tensor(x).cuda()).cpu().numpy()
    want, _ = MO.forward(net.params.cpu().numpy(), SMALL, x, shift, scale, emulate=True)
    np.testing.assert_allclose(y, want, rtol=1e-2, atol=2e-3)


@pytest.mark.gpu
def test_adam_with_the_step_on_the_device(cuda):
    """bmc_mlp_adam_step_dev: the same update as the host-step entry, and the count advanced."""
    torch = cuda
    a, b = _net(SMALL, seed=4), _net(SMALL, seed=4)
    rng = np.random.default_rng(9)
    g = torch.as_tensor(rng.normal(0, 1e-2, a.params.numel()).astype(np.float32)).cuda() * (a.params != 0)
    for net in (a, b):
        net.grad.copy_(g)
    a.step = 6
    a.adam(lr=1e-3)
    d_step = torch.tensor([6], dtype=torch.int32, device="cuda")
    b.adam_dev(d_step, lr=1e-3)
    assert int(d_step.item()) == 7
    np.testing.assert_allclose(b.params.cpu().numpy(), a.params.cpu().numpy(), rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(b.m.cpu().numpy(), a.m.cpu().numpy(), rtol=0, atol=0)


@pytest.mark.gpu
def test_graph_replayed_training_follows_the_eager_loop(cuda):
    """Training with the captured step takes the eager loop's steps (float atomics reorder sums: close,
    not equal)."""
    torch = cuda
    rng = np.random.default_rng(21)
    x = torch.as_tensor(rng.normal(0, 1, (8192, SMALL[0])).astype(np.float32)).cuda()
    t = torch.as_tensor(rng.normal(0, 0.5, (8192, SMALL[3])).astype(np.float32)).cuda()
    a, b = _net(SMALL, seed=5), _net(SMALL, seed=5)
    ha = a.train(x, t, epochs=3, batch=1024, lr=1e-3, seed=2, graph=True)
    hb = b.train(x, t, epochs=3, batch=1024, lr=1e-3, seed=2, graph=False)
    assert a.step == b.step == 24
    np.testing.assert_allclose(ha, hb, rtol=1e-3)
    np.testing.assert_allclose(a.params.cpu().numpy(), b.params.cpu().numpy(), rtol=1e-2, atol=1e-4)


@pytest.mark.gpu
def test_training_fits_a_teacher_network(cuda):
    """A student learns a random teacher's function: the loss falls by more than 10x."""
    torch = cuda
    teacher = MO.init_params(*SMALL, seed=11).astype(np.float64) * 3.0
    rng = np.random.default_rng(12)
    x = rng.normal(0, 1, (32768, SMALL[0])).astype(np.float32)
    t, _ = MO.forward(teacher, SMALL, x, emulate=False)
    net = _net(SMALL, seed=13)
    hist = net.train(torch.as_tensor(x).cuda(), torch.as_tensor(t.astype(np.float32)).cuda(), epochs=30,
                     batch=1024, lr=2e-3, seed=1)
    assert hist[-1] < 0.1 * hist[0], hist
