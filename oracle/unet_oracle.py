"""CPU oracle of the learned preconditioner's network (test infrastructure).

The checker for the U-Net kernels of libplategpu.so: the same architecture,
forward and backward passes, pooling, upsampling, Adam step and
energy-norm loss, written in numpy float64.  With ``bf16=True`` it rounds to
bfloat16 (round to nearest even) exactly where the GPU stores bfloat16
values -- network input, weights, every activation and every activation
gradient -- so a layer fed the same inputs agrees with the GPU up to FP32
accumulation order; with ``bf16=False`` it is plain float64, which the
finite-difference checks of the backward pass use.

The reference (cseifert512/gpu-gauntlet) has no learned preconditioner: its
PCG applies the 3x3 block-Jacobi preconditioner only
(src/lib/plate/gpu/shaders/index.ts:214-262, called from runGPUPCG in
src/lib/plate/gpu/solver.ts:190-553), which is where this network's
correction is added (two-level: block-Jacobi smoothing plus the network as
the coarse correction, inside flexible PCG).  Nothing here is imported by
the product; tests and the benchmark's checks use it.

Layout: activations [B][H][W][C] (channels last), weights [Cout][3][3][Cin]
(tap (dy, dx) with dy, dx in {0, 1, 2} meaning offsets -1, 0, +1), 3 x 3
convolutions with zero padding and no bias, ReLU after every convolution
but the last, 2 x 2 average pooling down, nearest-neighbour 2x upsampling,
and skip connections by channel concatenation [skip, upsampled].
"""
from __future__ import annotations

import numpy as np

# (name, cin, cout, relu) -- the input layer's 3 channels and the output
# layer's 3 channels are stored padded to 16 on the GPU (zero weights)
LAYERS = (
    ("e0a", 3, 16, True), ("e0b", 16, 16, True),
    ("e1a", 16, 32, True), ("e1b", 32, 32, True),
    ("e2a", 32, 64, True), ("e2b", 64, 64, True),
    ("e3a", 64, 128, True), ("e3b", 128, 128, True),
    ("d2a", 192, 64, True), ("d2b", 64, 64, True),
    ("d1a", 96, 32, True), ("d1b", 32, 32, True),
    ("d0a", 48, 16, True), ("d0b", 16, 16, True),
    ("out", 16, 3, False),
)
IN_CHANNELS = 3
OUT_CHANNELS = 3


def param_count():
    return sum(9 * ci * co for _n, ci, co, _r in LAYERS)


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) through float32; returns
    float64 values."""
    f = np.ascontiguousarray(np.asarray(x, np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def init_params(seed):
    """He-normal weights (std sqrt(2 / (9 cin))) in float64, drawn in layer
    order from numpy's default generator; the GPU network is initialised
    with the same values (set through pg_net_set_params)."""
    rng = np.random.default_rng(seed)
    out = []
    for _n, ci, co, relu in LAYERS:
        std = np.sqrt((2.0 if relu else 1.0) / (9.0 * ci))
        out.append(rng.standard_normal((co, 3, 3, ci)) * std)
    return out


def flatten(params):
    return np.concatenate([p.reshape(-1) for p in params])


def unflatten(flat):
    out, k = [], 0
    for _n, ci, co, _r in LAYERS:
        m = 9 * ci * co
        out.append(np.asarray(flat[k:k + m], np.float64).reshape(co, 3, 3, ci))
        k += m
    return out


def _pad(x):
    return np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))


def conv3x3(x, w):
    """y[b,i,j,o] = sum_{dy,dx,c} x[b,i+dy-1,j+dx-1,c] w[o,dy,dx,c]."""
    B, H, W, _ = x.shape
    xp = _pad(x)
    y = np.zeros((B, H, W, w.shape[0]))
    for dy in range(3):
        for dx in range(3):
            y += xp[:, dy:dy + H, dx:dx + W, :] @ w[:, dy, dx, :].T
    return y


def conv3x3_dgrad(g, w):
    """dL/dx of conv3x3 given g = dL/dy."""
    B, H, W, _ = g.shape
    gp = _pad(g)
    dx_ = np.zeros((B, H, W, w.shape[3]))
    for dy in range(3):
        for dx in range(3):
            # x[i] feeds y[i - dy + 1]
            dx_ += gp[:, 2 - dy:2 - dy + H, 2 - dx:2 - dx + W, :] @ w[:, dy, dx, :]
    return dx_


def conv3x3_wgrad(x, g):
    """dL/dw of conv3x3 given the input x and g = dL/dy."""
    B, H, W, C = x.shape
    xp = _pad(x)
    out = np.zeros((g.shape[3], 3, 3, C))
    gm = g.reshape(-1, g.shape[3])
    for dy in range(3):
        for dx in range(3):
            out[:, dy, dx, :] = gm.T @ xp[:, dy:dy + H, dx:dx + W, :].reshape(-1, C)
    return out


def pool2(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def up2(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def pool2_bwd(g):
    return up2(g) / 4.0


def up2_bwd(g):
    return 4.0 * pool2(g)


def forward(params, x, bf=False):
    """U-Net forward.  x: [B,H,W,3] (H, W multiples of 8).  Returns (out
    [B,H,W,3], cache for backward)."""
    r = bf16 if bf else (lambda a: a)
    W = [r(p) for p in params]
    c = {"x": r(x), "W": W, "bf": bf}

    def conv(name, k, inp, relu=True):
        z = conv3x3(inp, W[k])
        y = np.maximum(z, 0.0) if relu else z
        c[name] = r(y) if relu else y
        return c[name]

    e0a = conv("e0a", 0, c["x"])
    e0 = conv("e0", 1, e0a)
    p1 = c["p1"] = r(pool2(e0))
    e1a = conv("e1a", 2, p1)
    e1 = conv("e1", 3, e1a)
    p2 = c["p2"] = r(pool2(e1))
    e2a = conv("e2a", 4, p2)
    e2 = conv("e2", 5, e2a)
    p3 = c["p3"] = r(pool2(e2))
    e3a = conv("e3a", 6, p3)
    e3 = conv("e3", 7, e3a)
    cat2 = c["cat2"] = np.concatenate([e2, up2(e3)], axis=3)
    d2a = conv("d2a", 8, cat2)
    d2 = conv("d2", 9, d2a)
    cat1 = c["cat1"] = np.concatenate([e1, up2(d2)], axis=3)
    d1a = conv("d1a", 10, cat1)
    d1 = conv("d1", 11, d1a)
    cat0 = c["cat0"] = np.concatenate([e0, up2(d1)], axis=3)
    d0a = conv("d0a", 12, cat0)
    d0 = conv("d0", 13, d0a)
    out = conv("out", 14, d0, relu=False)
    return out, c


def backward(c, g_out):
    """Gradients of a scalar loss with dL/d(out) = g_out: returns (list of
    weight gradients in layer order, dL/dx)."""
    r = bf16 if c["bf"] else (lambda a: a)
    W = c["W"]
    gW = [None] * len(LAYERS)

    def mask(a):
        return (a > 0).astype(np.float64)

    def layer(k, inp, g, mask_input):
        """g = dL/dz of layer k; returns the (masked) gradient of its input."""
        gW[k] = conv3x3_wgrad(inp, g)
        d = conv3x3_dgrad(g, W[k])
        return r(d * mask(inp)) if mask_input else r(d)

    g = r(g_out)
    g = layer(14, c["d0"], g, True)          # dL/dz of d0
    g = layer(13, c["d0a"], g, True)
    dcat0 = layer(12, c["cat0"], g, True)
    C0 = c["e0"].shape[3]
    g = r(up2_bwd(dcat0[..., C0:]))          # dL/dz of d1
    g = layer(11, c["d1a"], g, True)
    dcat1 = layer(10, c["cat1"], g, True)
    C1 = c["e1"].shape[3]
    g = r(up2_bwd(dcat1[..., C1:]))          # d2
    g = layer(9, c["d2a"], g, True)
    dcat2 = layer(8, c["cat2"], g, True)
    C2 = c["e2"].shape[3]
    g = r(up2_bwd(dcat2[..., C2:]))          # e3
    g = layer(7, c["e3a"], g, True)
    dp3 = layer(6, c["p3"], g, False)
    g = r(dcat2[..., :C2] + pool2_bwd(dp3) * mask(c["e2"]))   # e2
    g = layer(5, c["e2a"], g, True)
    dp2 = layer(4, c["p2"], g, False)
    g = r(dcat1[..., :C1] + pool2_bwd(dp2) * mask(c["e1"]))   # e1
    g = layer(3, c["e1a"], g, True)
    dp1 = layer(2, c["p1"], g, False)
    g = r(dcat0[..., :C0] + pool2_bwd(dp1) * mask(c["e0"]))   # e0
    g = layer(1, c["e0a"], g, True)
    dx = layer(0, c["x"], g, False)
    return gW, dx


def adam(params, grads, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (t counts from 1) in float64; returns new (params, m, v)."""
    P, M, V = [], [], []
    for p, g, mm, vv in zip(params, grads, m, v):
        mm = b1 * mm + (1 - b1) * g
        vv = b2 * vv + (1 - b2) * g * g
        mh = mm / (1 - b1 ** t)
        vh = vv / (1 - b2 ** t)
        P.append(p - lr * mh / (np.sqrt(vh) + eps))
        M.append(mm)
        V.append(vv)
    return P, M, V


# --- the preconditioner around the network ---------------------------------------

def to_image(v, node_pixel, H, W, scale):
    """DOF vector [3 Nn] -> image [H, W, 3] (pixel node_pixel[n] gets node
    n's three values times scale; other pixels 0)."""
    img = np.zeros((H * W, 3))
    img[node_pixel] = v.reshape(-1, 3) * np.asarray(scale)[None, :]
    return img.reshape(H, W, 3)


def from_image(img, node_pixel, scale, cons):
    """image [H, W, 3] -> DOF vector, times scale, 0 on constrained DOFs."""
    v = (img.reshape(-1, 3)[node_pixel] * np.asarray(scale)[None, :]).reshape(-1)
    return np.where(np.asarray(cons) != 0, 0.0, v)


def block_apply(binv, v):
    Nn = binv.size // 9
    return np.einsum("nij,nj->ni", binv.reshape(Nn, 3, 3), v.reshape(Nn, 3)).reshape(-1)


def training_pair(A, binv, r, e):
    """The network's input and target for a residual/error pair (A e = r):
    pre-smoothing t = D^-1 r, r1 = r - A t, e1 = e - t (A e1 = r1)."""
    t = block_apply(binv, r)
    return r - A @ t, e - t


def energy_loss(A, e1, y):
    """(e1 - y)^T A (e1 - y) / e1^T A e1 and its gradient with respect to y."""
    d = e1 - y
    Ad = A @ d
    den = float(e1 @ (A @ e1))
    return float(d @ Ad) / den, -2.0 * Ad / den


def smoothed_energy_loss(A, binv, omega, e1, y, sweeps=2):
    """|M^nu (e1 - y)|_A^2 / |e1|_A^2 with M = I - omega D^-1 A: the energy
    norm of the error after the correction and `sweeps` damped block-Jacobi
    sweeps on it (the solve's smoothing of the network's correction)."""
    g = e1 - y
    for _ in range(sweeps):
        g = g - omega * block_apply(binv, A @ g)
    return float(g @ (A @ g)) / float(e1 @ (A @ e1))


def smoothed_energy_grad(A, binv, omega, e1, y, sweeps=2):
    """Gradient of smoothed_energy_loss with respect to y:
    -2 (M^T)^nu A M^nu (e1 - y) / |e1|_A^2, M^T = I - omega A D^-1."""
    g = e1 - y
    for _ in range(sweeps):
        g = g - omega * block_apply(binv, A @ g)
    h = A @ g
    for _ in range(sweeps):
        h = h - omega * (A @ block_apply(binv, h))
    return -2.0 * h / float(e1 @ (A @ e1))
