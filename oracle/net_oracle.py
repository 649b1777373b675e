"""CPU restatement of the damping network -- TEST INFRASTRUCTURE ONLY.

Used by tests/ to check the tensor-core forward and backward kernels of the
damping network (gnu_femlisp_b200/csrc/learn.cu); nothing in the product path
imports it.  The network has no counterpart in the reference (it is the
learned part added on top of Femlisp's <jacobi> smoother, linit.lisp:220-250),
so this restatement is pinned by finite differences of its own float64
gradient (tests/test_net_oracle.py) rather than by reference outputs.

With ``emulate=True`` the values the GPU rounds to BF16 -- input features,
weights, activations, the gradients fed to the tensor cores -- are rounded
here at the same points (round to nearest even); accumulation is float64,
so GPU and oracle differ only by FP32 accumulation order and the rare BF16
rounding flip that causes.

Layouts follow include/fmgpu.h: node order x fastest, flat parameters
W1[taps][32][16], b1[32], W2[taps][32][32], b2[32], W3[taps][32], b3[1],
tap = (dx+1) + 3(dy+1) (+ 9(dz+1)).
"""
from __future__ import annotations

import numpy as np

HID, NIN = 32, 16
OMEGA_MIN, OMEGA_MAX = 0.1, 1.3


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(a.shape)


def layout(dim: int) -> dict:
    taps = 27 if dim == 3 else 9
    o, L = 0, {"taps": taps}
    for name, size in (("w1", taps * HID * NIN), ("b1", HID), ("w2", taps * HID * HID), ("b2", HID),
                       ("w3", taps * HID), ("b3", 1)):
        L[name] = (o, o + size)
        o += size
    L["n"] = o
    return L


def unpack(p, dim: int, dtype=np.float32):
    L = layout(dim)
    t = L["taps"]
    g = lambda k: np.asarray(p[L[k][0]:L[k][1]], dtype=dtype)  # noqa: E731
    return (g("w1").reshape(t, HID, NIN), g("b1"), g("w2").reshape(t, HID, HID), g("b2"),
            g("w3").reshape(t, HID), g("b3"))


def shifts(dim: int):
    """(dz, dy, dx) of every tap in tap order."""
    out = []
    for t in range(27 if dim == 3 else 9):
        dx, dy = t % 3 - 1, (t // 3) % 3 - 1
        dz = t // 9 - 1 if dim == 3 else 0
        out.append((dz, dy, dx))
    return out


def _pad(a, dim):
    """zero ghost layer around the node axes of a [z][y][x][c] array (2D: no z padding)"""
    pz = (1, 1) if dim == 3 else (0, 0)
    return np.pad(a, (pz, (1, 1), (1, 1), (0, 0)))


def _window(ap, dim, s, shape):
    dz, dy, dx = s
    Z, Y, X = shape
    oz = 1 + dz if dim == 3 else 0
    return ap[oz:oz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X]


def conv(a, W, dim):
    """'same' convolution with zero padding: out[n][o] = sum_tap sum_i a[n + s(tap)][i] W[tap][o][i]
    (float64 accumulation)."""
    ap = _pad(a.astype(np.float64), dim)
    out = np.zeros(a.shape[:3] + (W.shape[1],))
    for t, s in enumerate(shifts(dim)):
        out += _window(ap, dim, s, a.shape[:3]) @ W[t].astype(np.float64).T
    return out


def conv_t(g, W, dim):
    """adjoint of conv in its input: out[n][i] = sum_tap sum_o g[n - s(tap)][o] W[tap][o][i]"""
    gp = _pad(g.astype(np.float64), dim)
    out = np.zeros(g.shape[:3] + (W.shape[2],))
    for t, s in enumerate(shifts(dim)):
        neg = tuple(-v for v in s)
        out += _window(gp, dim, neg, g.shape[:3]) @ W[t].astype(np.float64)
    return out


def wgrad(g, a, dim):
    """dW[tap][o][i] = sum_n g[n][o] a[n + s(tap)][i]"""
    ap = _pad(a.astype(np.float64), dim)
    G = g.reshape(-1, g.shape[-1]).astype(np.float64)
    out = []
    for s in shifts(dim):
        A = _window(ap, dim, s, g.shape[:3]).reshape(-1, a.shape[-1])
        out.append(G.T @ A)
    return np.stack(out)


def features(kcell, dim: int, n_top: int, level_n: int, emulate: bool = True):
    """Input channels of the nodes of a level with level_n cells per direction
    (learn.cu k_features): for each of the 2^dim cells around the node the
    mean over the cell's 2^dim Gauss points of log k (coefficient of the top
    level cell containing the point), centred by the mean log k over the top
    level cells and halved, clipped to [-8, 8]; then a presence bit per cell."""
    kc = np.asarray(kcell, dtype=np.float64)
    lk_top = np.log(kc)
    mu = lk_top.mean()
    ratio = n_top / level_n
    t = np.sqrt(1.0 / 3.0)
    xi = np.array([(1 + t) / 2, (1 - t) / 2])  # Gauss points (1 - t_k)/2 for t ascending
    top = lk_top.reshape((n_top,) * dim)       # [z][y][x] or [y][x]
    # mean log k per level cell over its Gauss points
    idx = [np.floor((np.arange(level_n)[:, None] + xi[None, :]) * ratio).astype(int)]  # [cell][q]
    f = idx[0]
    if dim == 2:
        cellv = sum(top[f[:, qy]][:, f[:, qx]] for qy in range(2) for qx in range(2)) / 4.0
    else:
        cellv = sum(top[f[:, qz]][:, f[:, qy]][:, :, f[:, qx]]
                    for qz in range(2) for qy in range(2) for qx in range(2)) / 8.0
    M = level_n + 1
    nc = 1 << dim
    X = np.zeros(((M if dim == 3 else 1), M, M, NIN), np.float64)
    for c in range(nc):
        bx, by, bz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        cx = np.arange(M) - 1 + bx
        cy = np.arange(M) - 1 + by
        okx = (cx >= 0) & (cx < level_n)
        oky = (cy >= 0) & (cy < level_n)
        if dim == 2:
            ok = oky[:, None] & okx[None, :]
            v = cellv[np.clip(cy, 0, level_n - 1)][:, np.clip(cx, 0, level_n - 1)]
            X[0, :, :, c] = np.where(ok, np.clip((v - mu) * 0.5, -8, 8), 0.0)
            X[0, :, :, nc + c] = ok
        else:
            cz = np.arange(M) - 1 + bz
            okz = (cz >= 0) & (cz < level_n)
            ok = okz[:, None, None] & oky[None, :, None] & okx[None, None, :]
            v = cellv[np.clip(cz, 0, level_n - 1)][:, np.clip(cy, 0, level_n - 1)][:, :, np.clip(cx, 0, level_n - 1)]
            X[:, :, :, c] = np.where(ok, np.clip((v - mu) * 0.5, -8, 8), 0.0)
            X[:, :, :, nc + c] = ok
    X = X.astype(np.float32)
    return bf16(X) if emulate else X.astype(np.float64)


def forward(p, X0, dim: int, emulate: bool = True):
    """Returns (omega [nodes], cache)."""
    W1, b1, W2, b2, W3, b3 = unpack(p, dim, np.float32 if emulate else np.float64)
    r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    W1r, W2r, W3r = r(W1), r(W2), r(W3)
    H1 = r(np.maximum(conv(X0, W1r, dim).astype(np.float32 if emulate else np.float64) + b1, 0))
    H2 = r(np.maximum(conv(H1, W2r, dim).astype(np.float32 if emulate else np.float64) + b2, 0))
    z = conv(H2, W3r[:, None, :], dim)[..., 0]
    z = z.astype(np.float32) + b3[0] if emulate else z + float(b3[0])
    s = 1.0 / (1.0 + np.exp(-np.asarray(z, np.float64)))
    omega = OMEGA_MIN + (OMEGA_MAX - OMEGA_MIN) * s
    cache = dict(X0=X0, H1=H1, H2=H2, W1=W1r, W2=W2r, W3=W3r, omega=omega)
    return omega.reshape(-1), cache


def backward(p, cache, gomega, dim: int, emulate: bool = True):
    """Gradient of sum(gomega * omega) with respect to the flat parameters."""
    L = layout(dim)
    r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    om = cache["omega"]
    g = np.asarray(gomega, np.float64).reshape(om.shape)
    dz = g * (om - OMEGA_MIN) * (OMEGA_MAX - om) / (OMEGA_MAX - OMEGA_MIN)
    dz = r(dz.astype(np.float32))[..., None] if emulate else dz[..., None]
    H1, H2, X0 = cache["H1"], cache["H2"], cache["X0"]
    out = np.zeros(L["n"])
    out[L["w3"][0]:L["w3"][1]] = wgrad(dz, H2, dim)[:, 0, :].ravel()
    out[L["b3"][0]] = dz.sum()
    dP2 = conv_t(dz, cache["W3"][:, None, :], dim) * (np.asarray(H2) > 0)
    dP2 = r(dP2.astype(np.float32)) if emulate else dP2
    out[L["w2"][0]:L["w2"][1]] = wgrad(dP2, H1, dim).ravel()
    out[L["b2"][0]:L["b2"][1]] = dP2.reshape(-1, HID).sum(0)
    dP1 = conv_t(dP2, cache["W2"], dim) * (np.asarray(H1) > 0)
    dP1 = r(dP1.astype(np.float32)) if emulate else dP1
    out[L["w1"][0]:L["w1"][1]] = wgrad(dP1, X0, dim).ravel()
    out[L["b1"][0]:L["b1"][1]] = dP1.reshape(-1, HID).sum(0)
    return out


def init_params(dim: int, seed: int = 0, scale: float = 1.0) -> np.ndarray:
    """Random parameters for tests (not the library's initialisation)."""
    L = layout(dim)
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1, 1, L["n"]).astype(np.float32)
    t = L["taps"]
    p[L["w1"][0]:L["w1"][1]] *= scale * np.sqrt(6.0 / (t * 2 ** (dim + 1)))
    p[L["w2"][0]:L["w2"][1]] *= scale * np.sqrt(6.0 / (t * HID))
    p[L["w3"][0]:L["w3"][1]] *= scale * np.sqrt(6.0 / (t * HID))
    p[L["b1"][0]:L["b1"][1]] *= 0.1
    p[L["b2"][0]:L["b2"][1]] *= 0.1
    return p
