"""CPU FP64 restatement of the surrogate network of include/sph_mlp.h (test
infrastructure: only the tests use it, as the checker of the GPU kernels).

The network has no reference counterpart; this file restates its definition: per head
z1 = W1 x + b1, h1 = GELU(z1), z2 = W2 h1 + b2, h2 = GELU(z2), z3 = W3 h2 + b3,
h3 = GELU(z3), out = W4 h3 + b4, loss = mean((out - y)^2) over the batch and outputs,
with exact GELU(z) = z/2 (1 + erf(z / sqrt 2)).  With bf16=True the weights, the
activations h1..h3 and the back-propagated dz1..dz3 are rounded to bf16 at the same points
as the GPU kernels (everything else in FP64), so the two differ only by FP32 versus FP64
accumulation; with bf16=False it is the plain FP64 network.
"""
import numpy as np
from scipy.special import erf

IN, HID, OUT = 6, 256, 4
SIZES = [("W1", HID * IN), ("b1", HID), ("W2", HID * HID), ("b2", HID), ("W3", HID * HID),
         ("b3", HID), ("W4", OUT * HID), ("b4", OUT)]
NPARAMS = sum(n for _, n in SIZES)
SHAPES = {"W1": (HID, IN), "W2": (HID, HID), "W3": (HID, HID), "W4": (OUT, HID)}


def offsets():
    out, o = {}, 0
    for name, n in SIZES:
        out[name] = (o, o + n)
        o += n
    return out


OFFS = offsets()


def bf16(a):
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    b = a32.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    t = {}
    for name, (a, b) in OFFS.items():
        v = np.asarray(p[a:b], dtype=np.float64)
        t[name] = v.reshape(SHAPES[name]) if name in SHAPES else v
    return t


def pack(t):
    return np.concatenate([np.ravel(t[name]) for name, _ in SIZES])


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(p, x, bf16_like_gpu=True):
    r = bf16 if bf16_like_gpu else (lambda a: np.asarray(a, dtype=np.float64))
    t = unpack(p)
    W = {k: r(t[k]) for k in ("W1", "W2", "W3", "W4")}
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W["W1"].T + t["b1"]
    h1 = r(gelu(z1))
    z2 = h1 @ W["W2"].T + t["b2"]
    h2 = r(gelu(z2))
    z3 = h2 @ W["W3"].T + t["b3"]
    h3 = r(gelu(z3))
    out = h3 @ W["W4"].T + t["b4"]
    return out, dict(W=W, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3, x=x)


def loss_and_grads(p, x, y, bf16_like_gpu=True):
    """Mean squared error and its gradient with respect to the packed parameters."""
    r = bf16 if bf16_like_gpu else (lambda a: np.asarray(a, dtype=np.float64))
    out, c = forward(p, x, bf16_like_gpu)
    y = np.asarray(y, dtype=np.float64)
    B = x.shape[0]
    loss = float(np.mean((out - y) ** 2))
    dout = 2.0 * (out - y) / (B * OUT)
    W = c["W"]
    g = {}
    g["W4"] = dout.T @ c["h3"]
    g["b4"] = dout.sum(0)
    dz3 = r((dout @ W["W4"]) * gelu_grad(c["z3"]))
    g["W3"] = dz3.T @ c["h2"]
    g["b3"] = dz3.sum(0)
    dz2 = r((dz3 @ W["W3"]) * gelu_grad(c["z2"]))
    g["W2"] = dz2.T @ c["h1"]
    g["b2"] = dz2.sum(0)
    dz1 = r((dz2 @ W["W2"]) * gelu_grad(c["z1"]))
    g["W1"] = dz1.T @ c["x"]
    g["b1"] = dz1.sum(0)
    return loss, pack(g)
