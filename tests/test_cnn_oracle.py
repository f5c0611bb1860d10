"""The CPU restatement of the learned warm start's network (oracle/cnn_oracle.py)
against finite differences: its backward pass is the gradient of its forward
pass (biases exactly, weights through their BF16 rounding)."""
import numpy as np


def test_oracle_gradient_matches_finite_differences():
    import cnn_oracle as co
    rng = np.random.default_rng(1)
    p = co.init_params(3, last_scale=1.0).astype(np.float64)
    x = rng.standard_normal((3, 6, 5))
    # the smooth network (hidden activations unrounded): finite differences
    y, _ = co.forward(p, x, tc_bf16=False)
    dy = rng.standard_normal(y.shape)
    g = co.backward(p, x, dy, tc_bf16=False)
    assert g.size == co.param_count() == 38177
    for k in (co.param_count() - 1, 864, 895, 896 + 9216 + 31):   # biases of layers 5, 0 and 1
        h = 1e-4
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = ((co.forward(pp, x, tc_bf16=False)[0] - co.forward(pm, x, tc_bf16=False)[0]) * dy).sum() / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])
    # the device's network rounds the hidden layers' operands to BF16 and
    # passes that rounding straight through its gradient: within a few BF16
    # ulps (2^-8) of the smooth network's
    g_tc = co.backward(p, x, dy, tc_bf16=True)
    assert np.linalg.norm(g_tc - g) <= 2e-2 * np.linalg.norm(g)
    assert not np.array_equal(g_tc, g)


def test_oracle_bf16_rounding():
    import cnn_oracle as co
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.1], dtype=np.float32)
    b = co.to_bf16(a)
    assert b[0] == 1.0 and b[1] == 1.0          # a tie rounds to even
    assert b[2] == np.float32(1.0078125)        # above the tie rounds up
    assert np.all((b.view(np.uint32) & 0xFFFF) == 0)
    assert np.all(np.abs(b - a) <= np.abs(a) * 2.0 ** -8)
