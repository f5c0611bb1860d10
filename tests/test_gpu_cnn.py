"""The learned warm start: the network's CUDA kernels against the CPU oracle
(oracle/cnn_oracle.py), training on the solver's own samples, and the warm
start in the solve against the same-stage warm start it is built on.

  one hidden layer on the       relative max error <= 1e-5 on BF16-exact inputs
  tensor cores                  (FP32 accumulation in tensor memory vs FP64)
  forward pass                  relative L2 error <= 3e-3
  parameter gradient            relative L2 error <= 2e-2
  mean-square loss and dy       <= 1e-6

The hidden layers take their operands in BF16; the device rounds its FP32
activations, the oracle its FP64 ones (through FP32), and a value near a
rounding boundary can round to neighbouring BF16 numbers in the two (a step
of 2^-8 relative), so the whole network agrees to a few 1e-4 and its
gradient, through the ReLU masks as well, to a few 1e-3; the single layer on
BF16-exact inputs isolates the tensor-core arithmetic itself.
  training                      the loss falls below that of predicting no change
  learned warm start            the fields stay within the pressure tolerance of
                                the plain path (1e-7 relative L2); the trained
                                network takes fewer pressure iterations than the
                                cold start (it does not beat the same-stage warm
                                start it is built on); both counts are reported
"""
import numpy as np
import pytest

from conftest import g_range, physical

pytestmark = pytest.mark.gpu


def test_tensor_core_layer_matches_oracle():
    """pvof_cnn_conv32: a 32 -> 32 layer as tcgen05 MMAs on BF16 operands,
    on pixel counts that are and are not multiples of the 128-pixel tile."""
    import torch
    import cnn_oracle as co
    from pvof.cnn import _ptr
    from pvof.runtime import check, load
    rng = np.random.default_rng(11)
    for H, W in ((16, 8), (13, 29), (70, 50)):
        x = co.to_bf16(rng.standard_normal((32, H, W)).astype(np.float32))
        w = co.to_bf16((rng.standard_normal((32, 32, 3, 3)) * 0.1).astype(np.float32))
        b = rng.standard_normal(32).astype(np.float32)
        wb = torch.tensor((w.view(np.uint32) >> 16).astype(np.int16).ravel(), device="cuda")
        xt = torch.tensor(x.ravel(), device="cuda")
        bt = torch.tensor(b, device="cuda")
        yt = torch.empty(32 * H * W, dtype=torch.float32, device="cuda")
        for relu in (0, 1):
            check(load().pvof_cnn_conv32(_ptr(xt), _ptr(wb), _ptr(bt), _ptr(yt), H, W, relu, None), "conv32")
            check(load().pvof_cnn_status(None), "status")
            ref = co.conv(x.astype(np.float64), w.astype(np.float64), b)
            if relu:
                ref = np.maximum(ref, 0.0)
            y = yt.cpu().numpy().reshape(32, H, W)
            assert np.abs(y - ref).max() <= 1e-5 * np.abs(ref).max(), (H, W, relu, np.abs(y - ref).max())


def test_network_kernels_match_oracle():
    import torch
    import cnn_oracle as co
    from pvof import cnn
    H, W = 20, 24
    rng = np.random.default_rng(3)
    p = co.init_params(5, last_scale=1.0)
    x = rng.standard_normal((3, H, W)).astype(np.float32)
    dy = rng.standard_normal((H, W)).astype(np.float32)
    net = cnn.Network(H, W, params=p)
    xt = torch.tensor(x.ravel(), device="cuda")
    y = net.forward(xt).cpu().numpy().reshape(H, W)
    net.status()
    y_ref, _ = co.forward(p, x)
    y_smooth, _ = co.forward(p, x, tc_bf16=False)
    err = np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref)
    assert err <= 3e-3, err
    # closer to the BF16-operand network than that is to the unrounded one
    assert err < np.linalg.norm(y_smooth - y_ref) / np.linalg.norm(y_ref)
    g = net.gradient(xt, torch.tensor(dy.ravel(), device="cuda")).cpu().numpy()
    net.status()
    g_ref = co.backward(p, x, dy)
    assert np.linalg.norm(g - g_ref) <= 2e-2 * np.linalg.norm(g_ref)
    # the loss kernel
    t = rng.standard_normal(H * W).astype(np.float32)
    loss_ref, dy_ref = co.mse(y.ravel(), t)
    net.loss.zero_()
    from pvof.runtime import check, load
    from pvof.cnn import _ptr
    tt = torch.tensor(t, device="cuda")
    check(load().pvof_cnn_mse(_ptr(net.y), _ptr(tt), _ptr(net.dy), H * W, _ptr(net.loss), net.stream), "mse")
    assert abs(net.loss.item() - loss_ref) <= 1e-6 * loss_ref
    assert np.abs(net.dy.cpu().numpy() - dy_ref).max() <= 1e-6 * np.abs(dy_ref).max()


def test_learned_warm_start_trains_and_stays_within_tolerance():
    from pvof import cases, cnn, runtime
    grid, params, planes = cases.rayleigh_taylor(64, 256, Lx=1.0, Ly=4.0, Cn=0.02, P_CG_MAXIT=2000)
    samples = cnn.generate_samples(grid, params, planes, 24, 1e-4)
    assert len(samples) == 66
    net, hist = cnn.train(samples[:54], grid.NYM, grid.NXM, epochs=25, batch=6, lr=2e-3)
    loss, base = net.evaluate(samples[:54])
    assert loss < base, (loss, base)
    P = net.params()
    out = {}
    for mode in (0, 1, 2):
        params.pressure_warm_start = mode
        s = runtime.Solver(grid, params, device=0)
        s.set_planes(planes)
        s.initialize()
        if mode == 2:
            s.set_pressure_network(P)
        iters = 0
        for n in range(24):
            for rk in range(3):
                if n > 0 and rk == 0:
                    s.call("Velocity_cell_center")
                s.set_stage(rk, 1e-4)
                iters += s.substep().p_iters_total
        out[mode] = (iters, {f: physical(grid, g_range(grid, s.get(f)), f) for f in ("U", "V", "P")})
        s.close()
    print("pressure iterations: cold %d, same-stage %d, learned %d; training loss %.3e vs no-change %.3e"
          % (out[0][0], out[1][0], out[2][0], loss, base))
    for mode in (1, 2):
        for f in ("U", "V", "P"):
            a, b = out[mode][1][f], out[0][1][f]
            assert np.linalg.norm(a - b) <= 1e-7 * np.linalg.norm(b), (mode, f)
    assert out[1][0] < out[0][0]
    # what the trained network gains over the Jacobi-PCG without a warm start
    assert out[2][0] < out[0][0], (out[2][0], out[0][0])
