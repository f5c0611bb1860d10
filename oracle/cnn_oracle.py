"""CPU restatement of the learned warm start's network (test infrastructure).

The same fixed network as parties-vof-ibm_b200/csrc/pvof_cnn.cu: six 3x3
convolutions 3 -> 32 -> 32 -> 32 -> 32 -> 32 -> 1 with zero padding and ReLU
between them; weights rounded to BF16 (round to nearest even) for the
forward and backward passes, biases in FP32; the four hidden 32 -> 32 layers
(TC_LAYERS, the tensor-core layers of the CUDA code) also take their input
activations, and in the backward pass their output gradient (the operand of
the input-gradient and weight-gradient GEMMs; the bias gradient sums it
unrounded), rounded to BF16 (through FP32, as the device holds them); here
every sum is in FP64.
Parameters are one flat array [w0, b0, ..., w5, b5], w_l laid out
[cout][cin][3][3]; planes are channel-major [C][H][W].

Only the tests use this module: it checks the CUDA forward pass, the
gradients of its backward pass and the loss.
"""
import numpy as np

CIN = 3
CMAX = 32
LAYERS = 6
TC_LAYERS = (1, 2, 3, 4)   # 32 -> 32: BF16 operands on the device's tensor cores


def shapes():
    out = []
    for l in range(LAYERS):
        ci = CIN if l == 0 else CMAX
        co = 1 if l == LAYERS - 1 else CMAX
        out.append((co, ci))
    return out


def param_count():
    return sum(co * ci * 9 + co for co, ci in shapes())


def unpack(params):
    """[(w (co, ci, 3, 3), b (co,)), ...] views of the flat array."""
    p = np.asarray(params)
    out, off = [], 0
    for co, ci in shapes():
        w = p[off:off + co * ci * 9].reshape(co, ci, 3, 3)
        off += co * ci * 9
        b = p[off:off + co]
        off += co
        out.append((w, b))
    return out


def bf16_operand(a):
    """An FP64 activation plane as the tensor cores take it: to FP32, then to
    the nearest BF16, back in FP64."""
    return to_bf16(np.asarray(a, dtype=np.float32)).astype(np.float64)


def to_bf16(a):
    """float32 -> nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + (((u >> 16) & 1) + 0x7FFF)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def init_params(seed=0, last_scale=0.0):
    """He-normal weights, zero biases; the last layer scaled by last_scale (0:
    the untrained network predicts no change)."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (co, ci) in enumerate(shapes()):
        w = rng.standard_normal((co, ci, 3, 3)) * np.sqrt(2.0 / (ci * 9))
        if l == LAYERS - 1:
            w = w * last_scale
        parts += [w.ravel(), np.zeros(co)]
    return np.concatenate(parts).astype(np.float32)


def conv(x, w, b):
    """3x3 convolution with zero padding; x (ci, H, W), w (co, ci, 3, 3)."""
    ci, H, W = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
    out = np.zeros((w.shape[0], H, W))
    for dy in range(3):
        for dx in range(3):
            out += np.einsum("oc,chw->ohw", w[:, :, dy, dx], xp[:, dy:dy + H, dx:dx + W])
    if b is not None:
        out += np.asarray(b, dtype=np.float64)[:, None, None]
    return out


def forward(params, x, tc_bf16=True):
    """Output (H, W) and the activations of every layer (after ReLU).
    tc_bf16=False keeps the hidden layers' activations unrounded (the smooth
    function whose gradient finite differences can check)."""
    acts = []
    a = np.asarray(x, dtype=np.float64)
    for l, (w, b) in enumerate(unpack(params)):
        a = conv(bf16_operand(a) if (tc_bf16 and l in TC_LAYERS) else a, to_bf16(w).astype(np.float64), b)
        if l < LAYERS - 1:
            a = np.maximum(a, 0.0)
        acts.append(a)
    return a[0], acts


def backward(params, x, dy, tc_bf16=True):
    """Gradient of sum(dy * y) with respect to the flat parameters; with
    tc_bf16 the device's: the BF16 rounding of the hidden layers' operands is
    passed straight through."""
    layers = unpack(params)
    _, acts = forward(params, x, tc_bf16)
    grads = [None] * LAYERS
    g = np.asarray(dy, dtype=np.float64)[None]
    for l in range(LAYERS - 1, -1, -1):
        w, _ = layers[l]
        wb = to_bf16(w).astype(np.float64)
        if l < LAYERS - 1:
            g = g * (acts[l] > 0.0)
        inp = np.asarray(x, dtype=np.float64) if l == 0 else acts[l - 1]
        if tc_bf16 and l in TC_LAYERS:
            inp = bf16_operand(inp)
        ci, H, W = inp.shape
        ip = np.pad(inp, ((0, 0), (1, 1), (1, 1)))
        gw = np.zeros(wb.shape)
        gg = bf16_operand(g) if (tc_bf16 and l in TC_LAYERS) else g   # the weight gradient's GEMM operand
        for dyy in range(3):
            for dxx in range(3):
                gw[:, :, dyy, dxx] = np.einsum("ohw,chw->oc", gg, ip[:, dyy:dyy + H, dxx:dxx + W])
        grads[l] = (gw, g.sum(axis=(1, 2)))
        if l > 0:   # the input gradient: the transposed convolution
            wt = wb[:, :, ::-1, ::-1].transpose(1, 0, 2, 3)
            g = conv(bf16_operand(g) if (tc_bf16 and l in TC_LAYERS) else g, wt, None)
    return np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])


def mse(y, t):
    y, t = np.asarray(y, dtype=np.float64), np.asarray(t, dtype=np.float64)
    e = y - t
    return float(np.mean(e * e)), 2.0 * e / e.size
