"""CPU reference of the warm-start convolutions (test oracle only).

3x3x3, stride 1, zero padding 1, channels-last activations (N, D, H, W, C) and
weights (Cout, 27, Cin) with tap t = (dz+1)*9 + (dy+1)*3 + (dx+1) -- the layout
of the library's tr_conv3d_* kernels -- computed in float64 with NumPy.
"""

import numpy as np


def conv3d(x, w, b=None):
    x = np.asarray(x, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    N, D, H, W, C = x.shape
    xp = np.zeros((N, D + 2, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1, 1:-1] = x
    y = np.zeros((N, D, H, W, w.shape[0]))
    for t in range(27):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        y += np.einsum("ndhwc,oc->ndhwo", xp[:, dz:dz + D, dy:dy + H, dx:dx + W], w[:, t, :])
    if b is not None:
        y += np.asarray(b, dtype=np.float64)
    return y


def conv3d_wgrad(x, gy):
    x = np.asarray(x, dtype=np.float64)
    gy = np.asarray(gy, dtype=np.float64)
    N, D, H, W, C = x.shape
    xp = np.zeros((N, D + 2, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1, 1:-1] = x
    dw = np.zeros((gy.shape[-1], 27, C))
    for t in range(27):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        dw[:, t, :] = np.einsum("ndhwo,ndhwc->oc", gy, xp[:, dz:dz + D, dy:dy + H, dx:dx + W])
    return dw


def conv3d_dgrad(gy, w):
    """Gradient w.r.t. the input: transpose of conv3d."""
    gy = np.asarray(gy, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    N, D, H, W, Co = gy.shape
    Ci = w.shape[2]
    gp = np.zeros((N, D + 2, H + 2, W + 2, Ci))
    for t in range(27):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        gp[:, dz:dz + D, dy:dy + H, dx:dx + W] += np.einsum("ndhwo,oc->ndhwc", gy, w[:, t, :])
    return gp[:, 1:-1, 1:-1, 1:-1]
