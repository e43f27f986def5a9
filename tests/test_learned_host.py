"""Host logic of the learned warm start without a GPU: argument checks of the i3g_unet_* C ABI
(made before any device call) and the training driver's bookkeeping (scales, learning-rate
schedule, mini-batches, summary) against a stub network."""
import ctypes as C

import numpy as np
import pytest


def _lib():
    from i3elvis_b200 import lib
    import os
    if not os.path.exists(lib.LIBPATH):
        from i3elvis_b200 import build
        build.build()
    from i3elvis_b200 import warmstart
    return warmstart._bind()


@pytest.mark.parametrize("dims", [(8, 9, 9), (9, 9, 10), (9, 13, 9), (1, 1, 1)])
def test_create_rejects_grids_the_levels_cannot_halve(dims):
    L = _lib()
    h = C.c_void_p()
    rc = L.i3g_unet_create(dims[0], dims[1], dims[2], 0, 1, C.byref(h))
    assert rc == -1
    assert not h.value
    assert b"n-1 divisible by 8" in L.i3g_last_error(None)


def test_null_arguments_are_rejected():
    L = _lib()
    assert L.i3g_unet_create(9, 9, 9, 0, 1, None) == -1
    n = C.c_int64()
    assert L.i3g_unet_nparams(None, C.byref(n)) == -1
    assert L.i3g_unet_train_step(None, None, 0, C.c_float(1e-3), None) == -1
    assert L.i3g_unet_predict(None, None) == -1
    assert L.i3g_stokes_guess_info(None, None, None, None, None) == -1
    L.i3g_unet_destroy(None)   # no-op


class StubNet:
    """Stands in for warmstart.UNet: samples in host memory, a loss that halves per step."""

    def __init__(self, n, samples):
        self.n = n
        self.samples = samples
        self.scales = None
        self.calls = []
        self.loss = 1.0

    def get_sample(self, slot):
        return self.samples[slot]

    def set_scales(self, *s):
        self.scales = s

    def train_step(self, slots, lr):
        self.calls.append((list(slots), lr))
        self.loss *= 0.5
        return self.loss


def test_fit_scales_and_training_schedule():
    from i3elvis_b200 import learned
    rng = np.random.default_rng(0)
    n = 64
    samples = []
    for _ in range(5):
        in5 = np.stack([rng.normal(21, 1.5, n), rng.normal(3300, 40, n), np.zeros(n), np.zeros(n), np.zeros(n)])
        tg4 = np.stack([rng.normal(0, 2e6, n)] + [rng.normal(0, 3e-10, n) for _ in range(3)])
        samples.append((in5.astype(np.float32), tg4.astype(np.float32)))
    net = StubNet(n, samples)
    sc = learned.fit_scales(net, range(5))
    le = np.concatenate([s[0][0] for s in samples]).astype(np.float64)
    assert np.isclose(sc[0], le.mean()) and np.isclose(sc[1], 1 / le.std())
    dv = np.concatenate([s[1][1:].ravel() for s in samples]).astype(np.float64)
    assert np.isclose(sc[4], np.sqrt(np.mean(dv ** 2)))
    assert np.isclose(sc[5], np.sqrt(np.mean(np.concatenate([s[1][0] for s in samples]).astype(np.float64) ** 2)))
    assert net.scales == sc
    hist = learned.train(net, list(range(5)), iters=11, batch=3, lr=1e-3)
    assert len(hist) == 11 and hist[-1] < hist[0]
    lrs = [lr for _, lr in net.calls]
    # cosine decay from lr to lr/10, batches of distinct slots
    assert np.isclose(lrs[0], 1e-3) and np.isclose(lrs[-1], 1e-4)
    assert all(a >= b for a, b in zip(lrs, lrs[1:]))
    assert all(len(set(b)) == 3 and set(b) <= set(range(5)) for b, _ in net.calls)


def test_summary_of_a_comparison():
    from i3elvis_b200 import learned
    rows = [dict(seed=s, step=0, default_cycles=20, learned_cycles=18, default_ms=10.0, learned_ms=9.0,
                 default_rel0=1e-2, learned_rel0=1e-3, rel_default=1e-2, rel_guess=1e-3, alpha=0.8, guess_used=1)
            for s in range(3)]
    rows.append(dict(seed=9, step=0, default_cycles=22, learned_cycles=22, default_ms=11.0, learned_ms=11.0,
                     default_rel0=1e-2, learned_rel0=1e-2, rel_default=1e-2, rel_guess=5e-2, alpha=0.0, guess_used=0))
    s = learned.summarize(rows)["step0"]
    assert s["cases"] == 4 and s["guess_used"] == 3
    assert s["default_cycles"] == 20.5 and s["learned_cycles"] == 19.0
    assert np.isclose(s["rel0_default"], 1e-2)
    assert np.isclose(s["rel0_learned_guess"], np.exp(np.mean(np.log([1e-3, 1e-3, 1e-3, 5e-2]))))
    assert s["alpha_median"] == 0.8
