"""CPU checks of the U-Net oracle (oracle/unet_ref.py): grid-transfer adjoints and the
backward pass against central finite differences of its own float64 forward pass.

The reference has no learned component, so this is what pins the oracle that the GPU
network is compared with (tests/test_gpu_unet.py)."""
import numpy as np

import unet_ref as U

DIMS = (9, 9, 9)
SCALES = (21.0, 0.5, 3300.0, 0.01, 1e-10, 1e6)


def sample(seed, dims=DIMS):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    in5 = np.stack([rng.uniform(19, 23, n), rng.uniform(3250, 3450, n), rng.normal(0, 1e-10, n),
                    rng.normal(0, 1e-10, n), rng.normal(0, 1e-10, n)]).astype(np.float32)
    tg4 = np.stack([rng.normal(0, 1e6, n), rng.normal(0, 1e-10, n), rng.normal(0, 1e-10, n),
                    rng.normal(0, 1e-10, n)]).astype(np.float32)
    return in5, tg4


def test_transfer_adjoints():
    rng = np.random.default_rng(3)
    f = rng.normal(size=(9, 17, 9, 3))
    c = rng.normal(size=(5, 9, 5, 3))
    # <P c, f> = 8 <c, R f>  (P^T = 8 R, R^T = P / 8)
    assert np.isclose(np.sum(U.prolong(c) * f), 8.0 * np.sum(c * U.restrict(f)), rtol=1e-12)
    # restriction of a constant interior field keeps it (away from the boundary)
    r = U.restrict(np.ones((9, 9, 9, 1)))
    assert np.allclose(r[1:-1, 1:-1, 1:-1], 1.0)
    assert np.allclose(U.prolong(np.ones((5, 5, 5, 1))), 1.0)


def test_conv_gradients_are_adjoint():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(5, 7, 5, 16))
    g = rng.normal(size=(5, 7, 5, 32))
    W = rng.normal(size=(27, 32, 16))
    # <conv(x, W), g> = <x, dgrad(g, W)> = <W, wgrad(x, g)>
    lhs = np.sum(U.conv3(x, W) * g)
    assert np.isclose(lhs, np.sum(x * U.conv3_dgrad(g, W)), rtol=1e-10)
    assert np.isclose(lhs, np.sum(W * U.conv3_wgrad(x, g)), rtol=1e-10)


def test_backward_matches_finite_differences():
    par = U.init_params(seed=5)
    in5, tg4 = sample(6)
    net = U.Net(par, DIMS, SCALES, round_bf16=False)
    loss, g = net.loss_grads(in5, tg4)
    assert loss > 0
    offs, n = U.param_offsets()
    rng = np.random.default_rng(7)
    checked = 0
    for li, (w, b) in enumerate(offs):
        cin, cout = U.layer_shapes()[li]
        cin_eff = U.IN_CH if li == 0 else cin
        # two weights (inside the real input channels) and one bias of every layer
        picks = []
        for _ in range(2):
            t, co, ci = rng.integers(27), rng.integers(cout), rng.integers(cin_eff)
            picks.append(w + (t * cout + co) * cin + ci)
        picks.append(b + rng.integers(cout))
        for k in picks:
            h = 1e-3 * max(abs(float(par[k])), 1e-2)
            pp, pm = par.astype(np.float64).copy(), par.astype(np.float64).copy()
            pp[k] += h
            pm[k] -= h
            lp, _ = U.Net(pp, DIMS, SCALES, round_bf16=False).loss_grads(in5, tg4)
            lm, _ = U.Net(pm, DIMS, SCALES, round_bf16=False).loss_grads(in5, tg4)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[k]) <= 2e-4 * max(abs(fd), abs(g[k])) + 1e-9 * loss, (li, k, fd, g[k])
            checked += 1
    assert checked == 3 * len(offs)
