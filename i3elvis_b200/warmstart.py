"""Learned warm start of the Stokes solve: ctypes binding of the ``i3g_unet_*`` C ABI.

The reference starts each Stokes solve from the previous step's v, P
(``move3mg.c:1969-2019``).  :class:`UNet` owns a 3-D U-Net on the GPU (``csrc/unet.cu``) that
maps log10 viscosity, density and that previous velocity to a correction of the start;
:meth:`UNet.predict` stages ``previous + correction`` for the context's next ``i3g_stokes``,
which keeps it only when its relative residual is lower than the default start's and then
iterates to the same tolerance.  Training data are recorded from the library's own solves
(:meth:`capture_input` before ``i3g_stokes``, :meth:`capture_target` after it).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib

P = C.c_void_p
_bound = False


def _bind():
    global _bound
    L = lib.load()
    if _bound:
        return L
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    dp = C.POINTER(C.c_double)
    L.i3g_unet_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(P)]
    L.i3g_unet_destroy.argtypes = [P]
    L.i3g_unet_destroy.restype = None
    L.i3g_unet_nparams.argtypes = [P, C.POINTER(C.c_int64)]
    L.i3g_unet_get_params.argtypes = [P, fp, C.c_int64]
    L.i3g_unet_set_params.argtypes = [P, fp, C.c_int64]
    L.i3g_unet_set_scales.argtypes = [P, fp]
    L.i3g_unet_set_sample.argtypes = [P, C.c_int, fp, fp]
    L.i3g_unet_get_sample.argtypes = [P, C.c_int, fp, fp]
    L.i3g_unet_capture_input.argtypes = [P, P, C.c_int]
    L.i3g_unet_capture_target.argtypes = [P, P, C.c_int]
    L.i3g_unet_train_step.argtypes = [P, ip, C.c_int, C.c_float, dp]
    L.i3g_unet_loss.argtypes = [P, ip, C.c_int, dp]
    L.i3g_unet_eval_host.argtypes = [P, fp, fp, fp, fp, dp]
    L.i3g_unet_predict.argtypes = [P, P]
    L.i3g_unet_time.argtypes = [P, C.c_int, dp, dp]
    L.i3g_unet_time_conv.argtypes = [P, C.c_int, C.c_int, dp, dp]
    u16 = C.POINTER(C.c_uint16)
    L.i3g_unet_conv_host.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, u16, u16, fp, u16, C.c_int, fp]
    L.i3g_unet_wgrad_host.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, u16, u16, fp, fp]
    L.i3g_stokes_guess_info.argtypes = [P, ip, dp, dp, dp]
    _bound = True
    return L


def _check(rc):
    if rc != 0:
        raise lib.I3gError(rc, lib.load().i3g_last_error(None).decode())


def _f32(a):
    a = np.ascontiguousarray(a, np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def conv_host(cin, cout, dims, x_bits, w_bits, bias=None, add_bits=None, relu=False):
    """One tensor-core convolution (``i3g_unet_conv_host``): BF16 bit patterns in, FP32 out
    [rows][cout] over the padded grid of ``dims = (nz, nx, ny)``."""
    L = _bind()
    nz, nx, ny = dims
    rows = (nz + 2) * (nx + 2) * (ny + 2)
    out = np.zeros((rows, cout), np.float32)
    u16 = C.POINTER(C.c_uint16)
    x = np.ascontiguousarray(x_bits, np.uint16)
    w = np.ascontiguousarray(w_bits, np.uint16)
    b = None if bias is None else np.ascontiguousarray(bias, np.float32)
    ad = None if add_bits is None else np.ascontiguousarray(add_bits, np.uint16)
    _check(L.i3g_unet_conv_host(cin, cout, nx, ny, nz, x.ctypes.data_as(u16), w.ctypes.data_as(u16),
                                None if b is None else b.ctypes.data_as(C.POINTER(C.c_float)),
                                None if ad is None else ad.ctypes.data_as(u16), int(relu),
                                out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def wgrad_host(cin, cout, dims, x_bits, g_bits):
    """Weight and bias gradients of one layer (``i3g_unet_wgrad_host``): BF16 bit patterns of the
    input [rows][cin] and of the output gradient [rows][cout] over the padded grid of
    ``dims = (nz, nx, ny)``; returns dW [27][cout][cin] and db [cout] (FP32)."""
    L = _bind()
    nz, nx, ny = dims
    u16 = C.POINTER(C.c_uint16)
    x = np.ascontiguousarray(x_bits, np.uint16)
    g = np.ascontiguousarray(g_bits, np.uint16)
    dw = np.zeros((27, cout, cin), np.float32)
    db = np.zeros(cout, np.float32)
    _check(L.i3g_unet_wgrad_host(cin, cout, nx, ny, nz, x.ctypes.data_as(u16), g.ctypes.data_as(u16),
                                 dw.ctypes.data_as(C.POINTER(C.c_float)), db.ctypes.data_as(C.POINTER(C.c_float))))
    return dw, db


def guess_info(ctx: lib.Context):
    """(used, rel_guess, rel_default, alpha) of the context's last Stokes solve."""
    L = _bind()
    u, a, b, al = C.c_int(), C.c_double(), C.c_double(), C.c_double()
    _check(L.i3g_stokes_guess_info(ctx.h, C.byref(u), C.byref(a), C.byref(b), C.byref(al)))
    return u.value, a.value, b.value, al.value


class UNet:
    """The network on the current GPU for a level-0 grid of ``nx x ny x nz`` nodes."""

    def __init__(self, nx, ny, nz, capacity=0, seed=1):
        L = _bind()
        self.h = P()
        self.dims = (nz, nx, ny)
        self.n = nx * ny * nz
        self.capacity = capacity
        _check(L.i3g_unet_create(nx, ny, nz, capacity, seed, C.byref(self.h)))
        n = C.c_int64()
        _check(L.i3g_unet_nparams(self.h, C.byref(n)))
        self.nparams = n.value
        self.scales = None

    def close(self):
        if getattr(self, "h", None):
            lib.load().i3g_unet_destroy(self.h)
            self.h = P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        out = np.zeros(self.nparams, np.float32)
        _check(_bind().i3g_unet_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), self.nparams))
        return out

    def set_params(self, par):
        a, p = _f32(par)
        _check(_bind().i3g_unet_set_params(self.h, p, a.size))

    def set_scales(self, eta_mean, eta_inv, ro_mean, ro_inv, v_scale, p_scale):
        self.scales = (eta_mean, eta_inv, ro_mean, ro_inv, v_scale, p_scale)
        a, p = _f32(self.scales)
        _check(_bind().i3g_unet_set_scales(self.h, p))

    def set_sample(self, slot, in5=None, tg4=None):
        L = _bind()
        a = b = None
        if in5 is not None:
            a, _ = _f32(in5)
        if tg4 is not None:
            b, _ = _f32(tg4)
        _check(L.i3g_unet_set_sample(self.h, slot, None if a is None else a.ctypes.data_as(C.POINTER(C.c_float)),
                                     None if b is None else b.ctypes.data_as(C.POINTER(C.c_float))))

    def get_sample(self, slot):
        in5 = np.zeros((5, self.n), np.float32)
        tg4 = np.zeros((4, self.n), np.float32)
        _check(_bind().i3g_unet_get_sample(self.h, slot, in5.ctypes.data_as(C.POINTER(C.c_float)),
                                           tg4.ctypes.data_as(C.POINTER(C.c_float))))
        return in5, tg4

    def capture_input(self, ctx: lib.Context, slot):
        _check(_bind().i3g_unet_capture_input(self.h, ctx.h, slot))

    def capture_target(self, ctx: lib.Context, slot):
        _check(_bind().i3g_unet_capture_target(self.h, ctx.h, slot))

    def train_step(self, slots, lr):
        s = np.ascontiguousarray(slots, np.int32)
        loss = C.c_double()
        _check(_bind().i3g_unet_train_step(self.h, s.ctypes.data_as(C.POINTER(C.c_int)), s.size, lr, C.byref(loss)))
        return loss.value

    def loss(self, slots):
        s = np.ascontiguousarray(slots, np.int32)
        loss = C.c_double()
        _check(_bind().i3g_unet_loss(self.h, s.ctypes.data_as(C.POINTER(C.c_int)), s.size, C.byref(loss)))
        return loss.value

    def eval_host(self, in5, tg4=None, grads=False):
        """(correction [4][n], loss or None, flat gradients or None) for host inputs."""
        L = _bind()
        a, pa = _f32(in5)
        out = np.zeros((4, self.n), np.float32)
        g = np.zeros(self.nparams, np.float32) if (grads and tg4 is not None) else None
        loss = C.c_double()
        if tg4 is not None:
            b, pb = _f32(tg4)
        else:
            pb = None
        _check(L.i3g_unet_eval_host(self.h, pa, pb, out.ctypes.data_as(C.POINTER(C.c_float)),
                                    None if g is None else g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return out, (loss.value if tg4 is not None else None), g

    def predict(self, ctx: lib.Context):
        _check(_bind().i3g_unet_predict(self.h, ctx.h))

    def time(self, reps=10):
        a, b = C.c_double(), C.c_double()
        _check(_bind().i3g_unet_time(self.h, reps, C.byref(a), C.byref(b)))
        return a.value, b.value

    def time_conv(self, layer, reps=20):
        """(ms per launch, algorithmic bytes) of one layer's forward convolution."""
        a, b = C.c_double(), C.c_double()
        _check(_bind().i3g_unet_time_conv(self.h, layer, reps, C.byref(a), C.byref(b)))
        return a.value, b.value
