"""CPU FP64 reference of the step-seeding network -- TEST INFRASTRUCTURE ONLY.

Forward and backward of the MLP the library trains (84 features -> 3 x 128 GELU -> 2,
mean-squared error), written with numpy in FP64.  With bf16=True it rounds operands to
bfloat16 (round to nearest even) at exactly the points where the GPU kernels feed the
tensor cores -- normalised inputs, weights, hidden activations, output gradient and
pre-activation gradients -- so its gradients are comparable to the kernels' at FP32
accumulation accuracy; with bf16=False it is the exact FP64 network.

Parameter layout (flat float vector, row-major [in][out] weights):
W1[96][128] (rows >= 84 zero), b1[128], W2[128][128], b2, W3[128][128], b3,
W4[128][8] (columns >= 2 zero), b4[8].
"""
import numpy as np
from scipy.special import erf

NIN, NFEAT, W, NOUT, NY = 96, 84, 128, 8, 2
SIZES = [("W1", NIN * W), ("b1", W), ("W2", W * W), ("b2", W), ("W3", W * W), ("b3", W), ("W4", W * NOUT),
         ("b4", NOUT)]


def unpack(p):
    out, o = {}, 0
    for name, n in SIZES:
        out[name] = np.asarray(p[o:o + n], dtype=np.float64)
        o += n
    out["W1"] = out["W1"].reshape(NIN, W)
    out["W2"] = out["W2"].reshape(W, W)
    out["W3"] = out["W3"].reshape(W, W)
    out["W4"] = out["W4"].reshape(W, NOUT)
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward_backward(p, xmean, xstd, X, T=None, bf=True):
    """Returns (Y [n][2], loss, grads flat) -- grads only when T is given."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    P = unpack(p)
    n = X.shape[0]
    xn = np.zeros((n, NIN))
    xn[:, :NFEAT] = (np.asarray(X, np.float32) - np.asarray(xmean, np.float32)[:NFEAT]) / \
        np.asarray(xstd, np.float32)[:NFEAT]
    a0 = r(xn)
    Ws = [r(P["W1"]), r(P["W2"]), r(P["W3"]), r(P["W4"])]
    bs = [P["b1"], P["b2"], P["b3"], P["b4"]]
    zs, hs = [], [a0]
    h = a0
    for l in range(3):
        z = h @ Ws[l] + bs[l]
        zs.append(z)
        h = r(gelu(z))
        hs.append(h)
    y = (h @ Ws[3] + bs[3])[:, :NY]
    if T is None:
        return y, None, None
    e = y - np.asarray(T, np.float64)
    loss = float((e * e).sum() / (n * NY))
    dy = np.zeros((n, NOUT))
    dy[:, :NY] = r(2.0 * e / (n * NY))
    g = {"W4": hs[3].T @ dy, "b4": dy.sum(0)}
    g["W4"][:, NY:] = 0.0
    g["b4"][NY:] = 0.0
    dh = dy @ Ws[3].T
    for l in (2, 1, 0):
        dz = r(dh * gelu_grad(zs[l]))
        g["W%d" % (l + 1)] = hs[l].T @ dz
        g["b%d" % (l + 1)] = dz.sum(0)
        dh = dz @ Ws[l].T
    g["W1"][NFEAT:, :] = 0.0
    return y, loss, pack(g)
