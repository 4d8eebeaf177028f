"""CPU reference of the scheduler's MLP (test infrastructure): the same
8 -> 32 -> 32 -> 6 ReLU network, parameter layout and masked MSE loss as the
device kernels, in float64, with analytic and finite-difference gradients."""
import numpy as np

NIN, NH, NOUT = 8, 32, 6
W1, B1 = 0, NIN * NH
W2 = B1 + NH
B2 = W2 + NH * NH
W3 = B2 + NH
B3 = W3 + NH * NOUT
NPARAMS = B3 + NOUT


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[W1:B1].reshape(NIN, NH), p[B1:W2], p[W2:B2].reshape(NH, NH), p[B2:W3],
            p[W3:B3].reshape(NH, NOUT), p[B3:NPARAMS])


def forward(p, X):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    h1 = np.maximum(X @ w1 + b1, 0)
    h2 = np.maximum(h1 @ w2 + b2, 0)
    return h1, h2, h2 @ w3 + b3


def loss(p, X, T):
    _, _, y = forward(p, X)
    T = np.asarray(T, np.float64)
    m = np.isfinite(T)
    d = np.where(m, y - np.where(m, T, 0), 0)
    return float((d ** 2).sum() / max(1, m.sum()))


def grad(p, X, T):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    h1, h2, y = forward(p, X)
    m = np.isfinite(T)
    dy = np.where(m, 2 * (y - np.where(m, T, 0)), 0) / max(1, m.sum())
    g = np.zeros(NPARAMS)
    g[W3:B3] = (h2.T @ dy).ravel()
    g[B3:NPARAMS] = dy.sum(0)
    dh2 = (dy @ w3.T) * (h2 > 0)
    g[W2:B2] = (h1.T @ dh2).ravel()
    g[B2:W3] = dh2.sum(0)
    dh1 = (dh2 @ w2.T) * (h1 > 0)
    g[W1:B1] = (X.T @ dh1).ravel()
    g[B1:W2] = dh1.sum(0)
    return g


def fd_grad(p, X, T, idx, eps=1e-6):
    out = []
    for i in idx:
        a = np.array(p, np.float64)
        b = a.copy()
        a[i] += eps
        b[i] -= eps
        out.append((loss(a, X, T) - loss(b, X, T)) / (2 * eps))
    return np.array(out)
