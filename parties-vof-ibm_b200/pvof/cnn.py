"""The learned warm start of the pressure solve: samples, training and use
of the network whose kernels are in csrc/pvof_cnn.cu, through the C ABI.

Samples come from the solver itself: with pressure_warm_start on, each
substep keeps its pressure correction per RK stage, and
pvof_pressure_network_sample returns, for a stage, the network inputs
(rho, rhs and the correction one step earlier, scaled) and the target (the
change of the correction, scaled).  Training runs the library's forward and
backward kernels and Adam on the GPU; PyTorch only provides the device
buffers and the stream.
"""
import ctypes as C

import numpy as np

from . import runtime
from .runtime import check, load


def param_count():
    return int(load().pvof_cnn_param_count())


def init_params(seed=0):
    """He-normal weights, zero biases, a zero last layer: the untrained
    network predicts no change, i.e. the same-stage warm start."""
    rng = np.random.default_rng(seed)
    parts = []
    shapes = [(32, 3)] + [(32, 32)] * 4 + [(1, 32)]
    for l, (co, ci) in enumerate(shapes):
        w = rng.standard_normal((co, ci, 3, 3)) * np.sqrt(2.0 / (ci * 9))
        if l == len(shapes) - 1:
            w = w * 0.0
        parts += [w.ravel(), np.zeros(co)]
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == param_count()
    return p


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Network:
    """Parameters, Adam state and work buffers on the device for H x W planes."""

    def __init__(self, H, W, params=None, seed=0, device=0):
        import torch
        self.torch = torch
        self.H, self.W = H, W
        self.dev = torch.device("cuda", device)
        n = param_count()
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        self.p = torch.tensor(p, dtype=torch.float32, device=self.dev)
        self.pb = torch.empty(n, dtype=torch.int16, device=self.dev)
        self.g = torch.zeros(n, dtype=torch.float32, device=self.dev)
        self.m = torch.zeros(n, dtype=torch.float32, device=self.dev)
        self.v = torch.zeros(n, dtype=torch.float32, device=self.dev)
        self.work = torch.empty(int(load().pvof_cnn_work_floats(H, W)), dtype=torch.float32, device=self.dev)
        self.y = torch.empty(H * W, dtype=torch.float32, device=self.dev)
        self.dy = torch.empty(H * W, dtype=torch.float32, device=self.dev)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.stream = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        self.step = 0
        check(load().pvof_cnn_to_bf16(_ptr(self.p), _ptr(self.pb), self.stream), "pvof_cnn_to_bf16")

    def forward(self, x):
        check(load().pvof_cnn_forward(_ptr(self.p), _ptr(self.pb), _ptr(x), _ptr(self.y), self.H, self.W,
                                      _ptr(self.work), self.stream), "pvof_cnn_forward")
        return self.y

    def status(self):
        """Raises if a tensor-core convolution since the last call gave up
        waiting for its matrix multiplications."""
        check(load().pvof_cnn_status(self.stream), "pvof_cnn_status")

    def gradient(self, x, dy):
        """Parameter gradient of sum(dy * y) at x (a fresh buffer)."""
        self.g.zero_()
        self.forward(x)
        check(load().pvof_cnn_backward(_ptr(self.p), _ptr(self.pb), _ptr(x), _ptr(dy), _ptr(self.g), self.H,
                                       self.W, _ptr(self.work), self.stream), "pvof_cnn_backward")
        return self.g.clone()

    def train_batch(self, batch, lr):
        """One Adam step on the mean loss of the (x, t) pairs; returns it."""
        self.g.zero_()
        self.loss.zero_()
        n = self.H * self.W
        for x, t in batch:
            self.forward(x)
            check(load().pvof_cnn_mse(_ptr(self.y), _ptr(t), _ptr(self.dy), n, _ptr(self.loss), self.stream),
                  "pvof_cnn_mse")
            self.dy.mul_(1.0 / len(batch))
            check(load().pvof_cnn_backward(_ptr(self.p), _ptr(self.pb), _ptr(x), _ptr(self.dy), _ptr(self.g),
                                           self.H, self.W, _ptr(self.work), self.stream), "pvof_cnn_backward")
        self.step += 1
        check(load().pvof_cnn_adam(_ptr(self.p), _ptr(self.g), _ptr(self.m), _ptr(self.v), _ptr(self.pb),
                                   self.step, lr, self.stream), "pvof_cnn_adam")
        return float(self.loss.item()) / len(batch)

    def evaluate(self, samples):
        """Mean loss over samples, and the loss of predicting no change."""
        tot = base = 0.0
        for x, t in samples:
            y = self.forward(x)
            tot += float(((y - t) ** 2).mean().item())
            base += float((t ** 2).mean().item())
        return tot / len(samples), base / len(samples)

    def params(self):
        return self.p.cpu().numpy().copy()


def generate_samples(grid, params, planes, nsteps, dt, device=0):
    """Run the case with the same-stage warm start and collect a (x, t) pair
    per substep from the third step on (the first two fill the kept
    corrections)."""
    import torch
    from . import abi
    p = abi.Params.from_buffer_copy(params)
    p.pressure_warm_start = 1
    s = runtime.Solver(grid, p, device=device)
    s.set_planes(planes)
    s.initialize()
    H, W = grid.NYM, grid.NXM
    dev = torch.device("cuda", device)
    out = []
    for n in range(nsteps):
        for rk in range(3):
            if n > 0 and rk == 0:
                s.call("Velocity_cell_center")
            s.set_stage(rk, dt)
            s.substep()
            if n >= 2:
                x = torch.empty(3 * H * W, dtype=torch.float32, device=dev)
                t = torch.empty(H * W, dtype=torch.float32, device=dev)
                check(load().pvof_pressure_network_sample(s.h, rk, _ptr(x), _ptr(t)), "pvof_pressure_network_sample")
                out.append((x, t))
    s.close()
    return out


def train(samples, H, W, epochs=30, batch=8, lr=1e-3, seed=0, device=0, log=None):
    """Train a fresh network on the samples; returns it and the loss history."""
    net = Network(H, W, seed=seed, device=device)
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        order = rng.permutation(len(samples))
        losses = []
        for q in range(0, len(order), batch):
            losses.append(net.train_batch([samples[k] for k in order[q:q + batch]], lr))
        hist.append(float(np.mean(losses)))
        if log:
            log("epoch %d loss %.4e" % (ep, hist[-1]))
    return net, hist


def crops(x, t, H, W, size, count, rng):
    """count random size x size windows of a full-plane sample (x: 3 planes,
    t: 1 plane, flat device tensors), as (x, t) pairs of flat tensors."""
    xs = x.view(3, H, W)
    ts = t.view(H, W)
    out = []
    for _ in range(count):
        j = int(rng.integers(0, H - size + 1))
        i = int(rng.integers(0, W - size + 1))
        out.append((xs[:, j:j + size, i:i + size].contiguous().view(-1), ts[j:j + size, i:i + size].contiguous().view(-1)))
    return out


def generate_crop_samples(grid, params, planes, particles, nsteps, dt, size, per_plane, seed=0, device=0, log=None):
    """Run the case (with resolved particles if given) with the same-stage
    warm start; from the third step on, every substep's full-plane sample
    gives per_plane random size x size crops."""
    import torch
    from . import abi
    p = abi.Params.from_buffer_copy(params)
    p.pressure_warm_start = 1
    s = runtime.Solver(grid, p, device=device)
    if particles:
        s.set_particles(particles)
        s.set_planes(dict(planes, C_L=planes["F"]))
    else:
        s.set_planes(planes)
    s.initialize()
    H, W = grid.NYM, grid.NXM
    dev = torch.device("cuda", device)
    rng = np.random.default_rng(seed)
    x = torch.empty(3 * H * W, dtype=torch.float32, device=dev)
    t = torch.empty(H * W, dtype=torch.float32, device=dev)
    out = []
    for n in range(nsteps):
        for rk in range(3):
            if n > 0 and rk == 0:
                s.call("Velocity_cell_center")
            s.set_stage(rk, dt)
            s.substep()
            if n >= 2:
                check(load().pvof_pressure_network_sample(s.h, rk, _ptr(x), _ptr(t)), "pvof_pressure_network_sample")
                out += crops(x, t, H, W, size, per_plane, rng)
        if log:
            log("sample step %d: %d crops" % (n, len(out)))
    s.close()
    return out
