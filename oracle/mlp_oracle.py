"""CPU oracle of the warm-start network (TEST INFRASTRUCTURE).

A numpy restatement of the forward and backward passes that the device
kernels (koral_b200/csrc/kgpu_mlp.cu) compute: BF16 rounding (round to
nearest even) of the inputs, weights and activations that enter a
tensor-core product, FP32 accumulation, SiLU, the mean squared error of the
standardised outputs.  Only the tests use it, to check the device forward
pass and gradients.
"""
import numpy as np

NIN, NH, NOUT, NOUTP = 16, 128, 7, 8
OW1 = 0
OB1 = OW1 + NIN * NH
OW2 = OB1 + NH
OB2 = OW2 + NH * NH
OW3 = OB2 + NH
OB3 = OW3 + NH * NOUTP
NPARAM = OB3 + NOUTP
OMEAN, OSCALE = NPARAM, NPARAM + NOUTP


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((a >> 16) & 1) + np.uint32(0x7FFF)
    return ((a + r) & np.uint32(0xFFFF0000)).view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(blob):
    b = np.asarray(blob, dtype=np.float32)
    return dict(W1=b[OW1:OB1].reshape(NIN, NH), b1=b[OB1:OW2], W2=b[OW2:OB2].reshape(NH, NH), b2=b[OB2:OW3],
                W3=b[OW3:OB3].reshape(NH, NOUTP), b3=b[OB3:NPARAM], mean=b[OMEAN:OMEAN + NOUTP],
                scale=b[OSCALE:OSCALE + NOUTP])


def forward(blob, X):
    """Standardised outputs and the intermediate values of the device pass."""
    p = unpack(blob)
    x = bf16(X)
    z1 = x @ bf16(p["W1"]) + p["b1"]
    a1 = bf16(silu(z1))
    z2 = a1 @ bf16(p["W2"]) + p["b2"]
    a2 = bf16(silu(z2))
    y = a2 @ bf16(p["W3"]) + p["b3"]
    return y, dict(x=x, z1=z1, a1=a1, z2=z2, a2=a2, p=p)


def predict(blob, X):
    """Unstandardised outputs, as kgpu_mlp_forward returns them."""
    y, c = forward(blob, X)
    return y * c["p"]["scale"] + c["p"]["mean"]


def gradient(blob, X, T):
    """Mean squared error of the standardised outputs over the batch and its
    gradient in the blob's layout (the first NPARAM entries)."""
    y, c = forward(blob, X)
    p = c["p"]
    n = X.shape[0]
    t = (np.asarray(T, np.float32) - p["mean"][:NOUT]) / p["scale"][:NOUT]
    e = np.zeros_like(y)
    e[:, :NOUT] = y[:, :NOUT] - t
    loss = float((e[:, :NOUT] ** 2).sum() / n)
    dy = 2.0 * e / n
    g = np.zeros(NPARAM, dtype=np.float64)
    g[OB3:NPARAM] = dy.sum(0)
    gw3 = c["a2"].T @ dy
    gw3[:, NOUT:] = 0.0
    g[OW3:OB3] = gw3.ravel()
    da2 = dy @ bf16(p["W3"]).T
    dz2 = bf16(da2 * dsilu(c["z2"]))
    g[OB2:OW3] = dz2.sum(0)
    g[OW2:OB2] = (c["a1"].T @ dz2).ravel()
    da1 = dz2 @ bf16(p["W2"]).T
    dz1 = da1 * dsilu(c["z1"])
    g[OB1:OW2] = dz1.sum(0)
    g[OW1:OB1] = (c["x"].T @ dz1).ravel()
    return loss, g
