"""FP64 numpy reference of the property MLP (1 -> 64 -> 64 -> 5, tanh).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA training kernels'
forward pass, loss and gradients.  The network has no counterpart in the
reference; it stands in for the table interpolation of THERM_PROP_UPDATE
(src/THERM_PROP_UPDATE.f90:129-205).

Parameter vector layout (float32 on the device, 4613 values):
  W1[64] b1[64] W2[64][64] (row = output unit) b2[64] W3[5][64] b3[5]
Input x = (h - h_mid) / h_half; outputs are the standardised residual
targets of (T, rho, mu, k, cp) over a least-squares degree-5 polynomial base
per output; loss = mean over samples and outputs of (y - t)^2.  The
normalisation vector is hmid, hhalf, mean[5], std[5], base[5][6] (powers of
x, lowest first), and the property is base_o(x) + mean_o + std_o * y_o.
"""
import numpy as np

NH, NO = 64, 5
NPARAM = NH + NH + NH * NH + NH + NO * NH + NO


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + NH]; o += NH
    b1 = p[o:o + NH]; o += NH
    W2 = p[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = p[o:o + NH]; o += NH
    W3 = p[o:o + NO * NH].reshape(NO, NH); o += NO * NH
    b3 = p[o:o + NO]; o += NO
    return W1, b1, W2, b2, W3, b3


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    a1 = np.tanh(np.outer(x, W1) + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    return a2 @ W3.T + b3, (a1, a2)


def loss_and_grad(p, x, t):
    """MSE loss and its gradient with respect to the parameter vector."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    y, (a1, a2) = forward(p, x)
    n = len(x)
    e = (y - t) * (2.0 / (n * NO))
    loss = float(np.mean((y - t) ** 2))
    gW3 = e.T @ a2
    gb3 = e.sum(0)
    d2 = (e @ W3) * (1 - a2 ** 2)
    gW2 = d2.T @ a1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1 - a1 ** 2)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    return loss, np.concatenate([gW1, gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])


NBASE = 6


def properties(p, norm, h):
    """FP64 model output (T, rho, mu, k, cp) at enthalpies h: polynomial base
    plus the de-standardised network residual."""
    norm = np.asarray(norm, dtype=np.float64)
    x = (np.asarray(h, dtype=np.float64) - norm[0]) / norm[1]
    y, _ = forward(p, x)
    mean, std = norm[2:2 + NO], norm[2 + NO:2 + 2 * NO]
    base = norm[2 + 2 * NO:].reshape(NO, NBASE)
    out = np.empty((len(x), NO))
    for o in range(NO):
        out[:, o] = np.polynomial.polynomial.polyval(x, base[o]) + mean[o] + std[o] * y[:, o]
    return out
