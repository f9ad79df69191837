"""ORACLE -- test infrastructure only.

NumPy (float64) restatement of the learned Newton-guess network of dynfd3dcuda_b200
(dfd_mlp.cu): forward pass, mean squared standardised error and its analytic gradient.
The GPU training kernels are checked against it; it is itself checked against central
finite differences (tests/test_mlp_oracle.py).  Only tests/ may import it.

Layout of the parameter vector: W1[32][4] b1[32] W2[32][32] b2[32] W3[32] b3 |
mu[4] sd[4] ymu ysd (1259 floats, the first 1249 trainable).
"""
import numpy as np

H = 32
OW1, OB1, OW2, OB2, OW3, OB3 = 0, 128, 160, 1184, 1216, 1248
NTRAIN, OMU, OSD, OYMU, OYSD, NPAR = 1249, 1249, 1253, 1257, 1258, 1259


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[OW1:OB1].reshape(H, 4), w[OB1:OW2], w[OW2:OB2].reshape(H, H), w[OB2:OW3], w[OW3:OB3], w[OB3],
            w[OMU:OSD], w[OSD:OYMU], w[OYMU], w[OYSD])


def forward(w, x):
    """Standardised network output for inputs x (n, 4), and the activations."""
    W1, b1, W2, b2, W3, b3, mu, sd, _, _ = unpack(w)
    xs = (np.asarray(x, np.float64) - mu) / sd
    h1 = np.tanh(xs @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3 + b3, (xs, h1, h2)


def predict(w, x):
    """De-standardised residual."""
    _, _, _, _, _, _, _, _, ym, ys = unpack(w)
    return forward(w, x)[0] * ys + ym


def loss_grad(w, x, y):
    """Mean squared standardised error and its gradient over the trainable weights."""
    W1, b1, W2, b2, W3, b3, mu, sd, ym, ys = unpack(w)
    out, (xs, h1, h2) = forward(w, x)
    yt = (np.asarray(y, np.float64) - ym) / ys
    e = out - yt
    n = len(e)
    loss = float((e * e).mean())
    go = 2.0 * e / n
    g = np.zeros(NTRAIN)
    g[OW3:OB3] = go @ h2
    g[OB3] = go.sum()
    d2 = go[:, None] * W3[None, :] * (1.0 - h2 * h2)
    g[OW2:OB2] = (d2.T @ h1).ravel()
    g[OB2:OW3] = d2.sum(0)
    d1 = (d2 @ W2) * (1.0 - h1 * h1)
    g[OW1:OB1] = (d1.T @ xs).ravel()
    g[OB1:OW2] = d1.sum(0)
    return loss, g
