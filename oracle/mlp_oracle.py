"""CPU restatement of the warm-start network (TEST INFRASTRUCTURE ONLY).

numpy FP64 forward and backward of the 16 -> 64 -> 64 -> 1 GELU (tanh form) network of
graphics_b200/csrc/sph_mlp.cu, with the same normalisation and, when
`bf16=True`, BF16 rounding at the points where the GPU kernels round (GEMM
operands: inputs, W1, W2, W3, H1, dZ2, dZ1).  Used to check the GPU forward
and backward kernels.  The network has no counterpart in the reference."""
import math

import numpy as np

NIN, NH = 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + NIN * NH
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NPARAM = OFF_B3 + 1

def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.asarray(x, np.float32).copy().view(np.uint32)
    a = (a + (((a >> 16) & 1) + np.uint32(0x7FFF))) & np.uint32(0xFFFF0000)
    return a.view(np.float32).astype(np.float64)


_C = math.sqrt(2.0 / math.pi)


def gelu(z):
    """GELU, tanh form: 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(_C * (z + 0.044715 * z ** 3)))


def gelu_d(z):
    t = np.tanh(_C * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _C * (1.0 + 3 * 0.044715 * z ** 2)


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[OFF_W1:OFF_B1].reshape(NIN, NH), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3], w[OFF_B3])


def forward(w, norm, X, rnd=bf16):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    r = rnd if rnd is not None else (lambda a: np.asarray(a, np.float64))
    mu, inv = norm[:NIN], norm[NIN:2 * NIN]
    x = r((np.asarray(X, np.float64) - mu) * inv)
    z1 = x @ r(W1) + b1
    h1 = r(gelu(z1))
    z2 = h1 @ r(W2) + b2
    y = gelu(z2) @ r(W3) + b3
    return dict(x=x, z1=z1, h1=h1, z2=z2, y=y)


def predict(w, norm, X, rnd=bf16):
    f = forward(w, norm, X, rnd)
    return f["y"] / norm[2 * NIN + 1] + norm[2 * NIN]


def gradient(w, norm, X, t, rnd=bf16):
    """(grad of mean squared error in normalised label units, loss)."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    r = rnd if rnd is not None else (lambda a: np.asarray(a, np.float64))
    f = forward(w, norm, X, rnd)
    tn = (np.asarray(t, np.float64) - norm[2 * NIN]) * norm[2 * NIN + 1]
    B = len(tn)
    err = f["y"] - tn
    g = 2.0 * err / B
    dW3 = gelu(f["z2"]).T @ g
    db3 = g.sum()
    dz2 = g[:, None] * r(W3)[None, :] * gelu_d(f["z2"])
    db2 = dz2.sum(0)
    dz2r = r(dz2)
    dh1 = dz2r @ r(W2).T
    dz1 = r(dh1 * gelu_d(f["z1"]))
    db1 = dz1.sum(0)
    dW2 = f["h1"].T @ dz2r
    dW1 = f["x"].T @ dz1
    out = np.zeros(NPARAM)
    out[OFF_W1:OFF_B1] = dW1.ravel()
    out[OFF_B1:OFF_W2] = db1
    out[OFF_W2:OFF_B2] = dW2.ravel()
    out[OFF_B2:OFF_W3] = db2
    out[OFF_W3:OFF_B3] = dW3
    out[OFF_B3] = db3
    return out, float(np.mean(err * err))
