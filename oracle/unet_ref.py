"""CPU oracle of the learned warm start's 3-D U-Net (TEST INFRASTRUCTURE ONLY).

Only ``tests/`` use this module, as the checker of the GPU network in
``i3elvis_b200/csrc/unet.cu``; the product never imports it.  The reference has no learned
component (its Stokes solve starts from the previous step, ``move3mg.c:1969-2019``), so this
oracle is pinned by finite differences of its own float64 forward pass
(``tests/test_unet_oracle.py``) rather than by reference outputs.

Arrays are nodal, channels-last ``[nz, nx, ny, C]`` (the solver's node order, y fastest).
With ``bf16=True`` every stored tensor is rounded to bfloat16 (round to nearest even) at the
same points as the GPU network: inputs, weights, every activation and every activation
gradient; accumulation is float64 here and FP32 on the GPU.
"""
from __future__ import annotations

import numpy as np

CH = (16, 32, 64, 128)
IN_CH, OUT_CH = 5, 4

# tensors and layers in the order of unet.cu: name -> (level, channels)
TENSORS = dict(x0=(0, 16), e0a=(0, 16), e0=(0, 16), d1=(1, 16), e1a=(1, 32), e1=(1, 32), d2=(2, 32),
               e2a=(2, 64), e2=(2, 64), d3=(3, 64), b3a=(3, 128), b3=(3, 128), u2=(2, 128), g2a=(2, 64),
               g2=(2, 64), u1=(1, 64), g1a=(1, 32), g1=(1, 32), u0=(0, 32), g0a=(0, 16), g0=(0, 16), y=(0, 16))
LAYERS = [("x0", "e0a", None, True), ("e0a", "e0", None, True), ("d1", "e1a", None, True), ("e1a", "e1", None, True),
          ("d2", "e2a", None, True), ("e2a", "e2", None, True), ("d3", "b3a", None, True), ("b3a", "b3", None, True),
          ("u2", "g2a", "e2", True), ("g2a", "g2", None, True), ("u1", "g1a", "e1", True), ("g1a", "g1", None, True),
          ("u0", "g0a", "e0", True), ("g0a", "g0", None, True), ("g0", "y", None, False)]
DOWN = {"d1": "e0", "d2": "e1", "d3": "e2"}      # restriction inputs
UP = {"u2": "b3", "u1": "g2", "u0": "g1"}        # prolongation inputs
SKIP_OF_DOWN = {"d1": "g0a", "d2": "g1a", "d3": "g2a"}


def bf16(a):
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    b = f.view(np.uint32)
    r = ((b >> 16) & 1) + np.uint32(0x7FFF)
    out = ((b + r) & np.uint32(0xFFFF0000)).astype(np.uint32)
    return out.view(np.float32).astype(np.float64)


def bf16_bits(a):
    """bfloat16 bit patterns (uint16) of a, rounded to nearest even."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    b = f.view(np.uint32)
    r = ((b >> 16) & 1) + np.uint32(0x7FFF)
    return ((b + r) >> 16).astype(np.uint16)


def layer_shapes():
    return [(TENSORS[i][1], TENSORS[o][1]) for i, o, _, _ in LAYERS]


def param_offsets():
    """Offsets of W [27][cout][cin] and b [cout] of every layer in the flat parameter array."""
    offs, n = [], 0
    for cin, cout in layer_shapes():
        w = n
        n += 27 * cin * cout
        offs.append((w, n))
        n += cout
    return offs, n


def unflatten(par):
    offs, _ = param_offsets()
    out = []
    for (cin, cout), (w, b) in zip(layer_shapes(), offs):
        out.append((par[w:w + 27 * cin * cout].reshape(27, cout, cin).astype(np.float64),
                    par[b:b + cout].astype(np.float64)))
    return out


def level_dims(nz, nx, ny, lev):
    s = 1 << lev
    return ((nz - 1) // s + 1, (nx - 1) // s + 1, (ny - 1) // s + 1)


def _pad(x):
    return np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))


def conv3(x, W, b=None):
    """3x3x3 convolution with zero padding: out[p, co] = sum_tap,ci W[tap, co, ci] x[p+d_tap, ci] (+ b)."""
    nz, nx, ny, _ = x.shape
    xp = _pad(x)
    out = np.zeros((nz, nx, ny, W.shape[1]))
    t = 0
    for dz in (-1, 0, 1):
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                sh = xp[1 + dz:1 + dz + nz, 1 + dx:1 + dx + nx, 1 + dy:1 + dy + ny]
                out += sh @ W[t].T
                t += 1
    if b is not None:
        out += b
    return out


def conv3_wgrad(x, g):
    """dW[tap, co, ci] = sum_p g[p, co] x[p + d_tap, ci]."""
    nz, nx, ny, cin = x.shape
    xp = _pad(x)
    gw = np.zeros((27, g.shape[3], cin))
    G = g.reshape(-1, g.shape[3])
    t = 0
    for dz in (-1, 0, 1):
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                sh = xp[1 + dz:1 + dz + nz, 1 + dx:1 + dx + nx, 1 + dy:1 + dy + ny].reshape(-1, cin)
                gw[t] = G.T @ sh
                t += 1
    return gw


def conv3_dgrad(g, W):
    """Input gradient: dx[p, ci] = sum_tap,co W[tap, co, ci] g[p - d_tap, co] (the flipped transposed conv)."""
    Wt = np.transpose(W[::-1], (0, 2, 1))   # [26-tap][ci][co]
    return conv3(g, Wt)


def restrict(x):
    """Full weighting to the next coarser vertex-centred level (weights 1/4, 1/2, 1/4 per axis)."""
    out = x
    for ax in range(3):
        n = out.shape[ax]
        nc = (n - 1) // 2 + 1
        idx = np.arange(nc) * 2
        c = 0.5 * np.take(out, idx, axis=ax)
        lo = idx - 1
        hi = idx + 1
        vlo = np.take(out, np.clip(lo, 0, n - 1), axis=ax)
        vhi = np.take(out, np.clip(hi, 0, n - 1), axis=ax)
        shape = [1] * out.ndim
        shape[ax] = nc
        c = c + 0.25 * vlo * (lo >= 0).reshape(shape) + 0.25 * vhi * (hi <= n - 1).reshape(shape)
        out = c
    return out


def prolong(x):
    """Trilinear interpolation to the next finer vertex-centred level (P^T = 8 R, R^T = P / 8)."""
    out = x
    for ax in range(3):
        nc = out.shape[ax]
        nf = 2 * nc - 1
        f = np.arange(nf)
        a = np.take(out, f // 2, axis=ax)
        b = np.take(out, np.minimum(f // 2 + 1, nc - 1), axis=ax)
        shape = [1] * out.ndim
        shape[ax] = nf
        odd = (f % 2 == 1).reshape(shape)
        out = np.where(odd, 0.5 * (a + b), a)
    return out


def pack_input(in5, dims, scales):
    """in5 [5][n] (log10 eta, rho, vx, vy, vz) -> x0 [nz, nx, ny, 16] scaled."""
    nz, nx, ny = dims
    eta_mean, eta_inv, ro_mean, ro_inv, v_scale, p_scale = [np.float32(s) for s in scales]
    iv = np.float32(1.0) / v_scale
    x = np.zeros((nz, nx, ny, 16), np.float32)
    f = [(in5[0].astype(np.float32) - eta_mean) * eta_inv, (in5[1].astype(np.float32) - ro_mean) * ro_inv,
         in5[2].astype(np.float32) * iv, in5[3].astype(np.float32) * iv, in5[4].astype(np.float32) * iv]
    for c in range(5):
        x[..., c] = f[c].reshape(nz, nx, ny)
    return x.astype(np.float64)


class Net:
    """Forward and backward of the network with float64 accumulation."""

    def __init__(self, par, dims, scales, round_bf16=True):
        self.layers = unflatten(np.asarray(par, np.float32))
        self.dims = dims
        self.scales = scales
        self.r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
        self.Wq = [(self.r(W), b) for W, b in self.layers]

    def forward(self, in5):
        r = self.r
        A = {"x0": r(pack_input(in5, self.dims, self.scales))}
        for li, (i, o, add, relu) in enumerate(LAYERS):
            if i in DOWN:
                A[i] = r(restrict(A[DOWN[i]]))
            elif i in UP:
                A[i] = r(prolong(A[UP[i]]))
            W, b = self.Wq[li]
            z = conv3(A[i], W, b)
            if add:
                z = z + A[add]
            A[o] = r(np.maximum(z, 0.0) if relu else z)
        self.A = A
        return A["y"]

    def output(self, in5):
        """Correction [4][n] in physical units."""
        y = self.forward(in5)
        s = self.scales
        sc = np.array([s[5], s[4], s[4], s[4]], np.float64)
        return (y[..., :4] * sc).reshape(-1, 4).T

    def loss_grads(self, in5, tg4):
        """Loss (mean over nodes and 4 outputs of (y - t/scale)^2) and flat parameter gradients."""
        r = self.r
        y = self.forward(in5)
        A = self.A
        s = self.scales
        inv = np.array([1 / np.float32(s[5]), 1 / np.float32(s[4]), 1 / np.float32(s[4]), 1 / np.float32(s[4])])
        nz, nx, ny = self.dims
        n = nz * nx * ny
        t = (tg4.T.astype(np.float64) * inv).reshape(nz, nx, ny, 4)
        d = y[..., :4] - t
        loss = float(np.sum(d * d) / (4 * n))
        G = {}
        gy = np.zeros_like(y)
        gy[..., :4] = 2.0 * d / (4 * n)
        G["y"] = r(gy)
        grads = [None] * len(LAYERS)
        relu_out = {o for _, o, _, rl in LAYERS if rl}
        for li in range(len(LAYERS) - 1, -1, -1):
            i, o, add, relu = LAYERS[li]
            W, b = self.Wq[li]
            gz = G[o]
            grads[li] = (conv3_wgrad(A[i], gz), gz.sum(axis=(0, 1, 2)))
            if li == 0:
                break
            gi = conv3_dgrad(gz, W)
            if i in relu_out:
                gi = gi * (A[i] > 0)
            G[i] = r(gi)
            if i in UP:
                src = UP[i]
                G[src] = r(8.0 * restrict(G[i]) * (A[src] > 0))
            elif i in DOWN:
                src = DOWN[i]
                G[src] = r((prolong(G[i]) / 8.0 + G[SKIP_OF_DOWN[i]]) * (A[src] > 0))
        offs, ntot = param_offsets()
        flat = np.zeros(ntot)
        for (w, bo), (gw, gb) in zip(offs, grads):
            flat[w:w + gw.size] = gw.reshape(-1)
            flat[bo:bo + gb.size] = gb
        return loss, flat


def init_params(seed=1):
    """A random parameter vector (He-style scale) for tests."""
    rng = np.random.default_rng(seed)
    offs, n = param_offsets()
    par = np.zeros(n, np.float32)
    for li, ((cin, cout), (w, b)) in enumerate(zip(layer_shapes(), offs)):
        cin_eff = IN_CH if li == 0 else cin
        W = rng.normal(0, np.sqrt(2.0 / (27 * cin_eff)), size=(27, cout, cin)).astype(np.float32)
        if li == 0:
            W[:, :, IN_CH:] = 0
        par[w:w + W.size] = W.reshape(-1)
        par[b:b + cout] = rng.normal(0, 0.05, size=cout)
    return par
