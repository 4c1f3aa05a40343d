"""CPU restatement of the learned starting iterate's network, for tests only.

Test infrastructure: the product never imports this module.  It restates, in
numpy, the forward pass and the gradient that torch_b200/csrc/mlp.cu computes
on the tensor cores, with the same parameter layout (W1[5][64] b1[64]
W2[64][64] b2[64] W3[64][3] b3[3], then input mean/scale and output
mean/scale) and, when `emulate` is set, the same rounding points: the
normalised inputs, the hidden activations, dY and dZ2 are rounded to BF16
(round to nearest even) where the GPU hands them to the tensor cores, and the
weights are the BF16 images of the FP32 parameters.  Accumulation here is
FP64, so GPU and oracle differ by FP32 accumulation order and by the rare BF16
rounding that this flips.  With `emulate` off everything is FP64 (for the
finite-difference check of the gradient formulas themselves).

The network has no counterpart in the reference (its implicit solve,
src/Radiation/Radiation.cpp:375-478, starts from the current x_HII); what is
pinned here is the GPU's arithmetic against this statement of it.
"""
import numpy as np

IN, HID, OUT = 5, 64, 3
NTRAIN = IN * HID + HID + HID * HID + HID + HID * OUT + OUT
NPARAMS = NTRAIN + 2 * IN + 2 * OUT


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p, dtype=np.float32):
    p = np.asarray(p, dtype=dtype)
    o = 0

    def take(n, shape=None):
        nonlocal o
        v = p[o:o + n]
        o += n
        return v.reshape(shape) if shape else v
    d = {}
    d["W1"] = take(IN * HID, (IN, HID))
    d["b1"] = take(HID)
    d["W2"] = take(HID * HID, (HID, HID))
    d["b2"] = take(HID)
    d["W3"] = take(HID * OUT, (HID, OUT))
    d["b3"] = take(OUT)
    d["in_mean"] = take(IN)
    d["in_scale"] = take(IN)
    d["out_mean"] = take(OUT)
    d["out_scale"] = take(OUT)
    return d


def _round(x, emulate):
    return bf16(x).astype(np.float64) if emulate else np.asarray(x, dtype=np.float64)


def _layers(d, emulate):
    W = {k: _round(d[k], emulate) for k in ("W1", "W2", "W3")}
    b = {k: np.asarray(d[k], dtype=np.float32 if emulate else np.float64).astype(np.float64)
         for k in ("b1", "b2", "b3")}
    return W, b


def _f32(x, emulate):
    return np.asarray(x, dtype=np.float32).astype(np.float64) if emulate else x


def forward(p, x_raw, emulate=True):
    """Raw outputs [n x 3] for raw inputs [n x 5] (mlp.cu: infer_tile)."""
    d = unpack(p, np.float32 if emulate else np.float64)
    W, b = _layers(d, emulate)
    x = np.asarray(x_raw, dtype=np.float32 if emulate else np.float64)
    if emulate:
        xn = ((x - d["in_mean"]) * d["in_scale"]).astype(np.float32)
    else:
        xn = (x - d["in_mean"].astype(np.float64)) * d["in_scale"].astype(np.float64)
    xb = _round(xn, emulate)
    h1 = _round(np.maximum(_f32(xb @ W["W1"] + b["b1"], emulate), 0.0), emulate)
    h2 = _round(np.maximum(_f32(h1 @ W["W2"] + b["b2"], emulate), 0.0), emulate)
    y = _f32(h2 @ W["W3"] + b["b3"], emulate)
    return y / d["out_scale"].astype(np.float64) + d["out_mean"].astype(np.float64)


def gradient(p, records, out_weight, emulate=True):
    """(summed gradient [NTRAIN], loss) of 1/2 sum w (y - t)^2 over the
    records [n x 8] in normalised target units (mlp.cu: k_mlp_grad)."""
    d = unpack(p, np.float32 if emulate else np.float64)
    W, b = _layers(d, emulate)
    r = np.asarray(records, dtype=np.float32 if emulate else np.float64)
    w = np.asarray(out_weight, dtype=np.float64)
    if emulate:
        xn = ((r[:, :IN] - d["in_mean"]) * d["in_scale"]).astype(np.float32)
        tg = ((r[:, IN:] - d["out_mean"]) * d["out_scale"]).astype(np.float32).astype(np.float64)
    else:
        xn = (r[:, :IN] - d["in_mean"].astype(np.float64)) * d["in_scale"].astype(np.float64)
        tg = (r[:, IN:] - d["out_mean"].astype(np.float64)) * d["out_scale"].astype(np.float64)
    x = _round(xn, emulate)
    h1 = _round(np.maximum(_f32(x @ W["W1"] + b["b1"], emulate), 0.0), emulate)
    h2 = _round(np.maximum(_f32(h1 @ W["W2"] + b["b2"], emulate), 0.0), emulate)
    y = _f32(h2 @ W["W3"] + b["b3"], emulate)
    e = y - tg
    loss = 0.5 * float(np.sum(w * e * e))
    dy = _f32(w * e, emulate)
    dyb = _round(dy, emulate)
    dz2 = np.where(h2 > 0, _f32(dyb @ W["W3"].T, emulate), 0.0)
    dz2b = _round(dz2, emulate)
    dz1 = np.where(h1 > 0, _f32(dz2b @ W["W2"].T, emulate), 0.0)
    g = np.concatenate([
        (x.T @ dz1).ravel(), dz1.sum(0),
        (h1.T @ dz2b).ravel(), dz2.sum(0),
        (h2.T @ dyb).ravel(), dy.sum(0),
    ])
    return g, loss
