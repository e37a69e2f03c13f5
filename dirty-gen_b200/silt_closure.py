"""Host side of the learned sub-grid flux closure (include/silt_closure.h).

The network, its tensor-core kernels and the closure step live in
libsilt_b200.so; this module binds them for torch tensors (device memory and
streams only: every convolution, gradient and update runs in the library's
own kernels) and holds the training loop that fits the closure to pairs the
nested 2 cm sheets generate.

Shapes: activations NHWC BF16 [image, row, col, channel]; parameters one FP32
vector in the order of SILT_CLOSURE_NPARAM (W1 [9][16][32], b1, W2 [9][32][32],
b2, W3 [9][32][16], b3; weights [tap][cin][cout], tap = 3 (dy + 1) + (dx + 1)).
"""
import ctypes

import numpy as np

import silt_b200

CROP = 32
CIN, HID, COUT = 16, 32, 16
IN_USED, OUT_USED = 6, 8
NPARAM = 9 * CIN * HID + HID + 9 * HID * HID + HID + 9 * HID * COUT + COUT
NNORM = 20
COUPLING_NESTED, COUPLING_NONE, COUPLING_CLOSURE = 0, 1, 2

# (name, cin, cout) of the three layers, in parameter order.
LAYERS = (("1", CIN, HID), ("2", HID, HID), ("3", HID, COUT))

_p, _i, _f = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float


class ClosureStats(ctypes.Structure):
    _fields_ = [("closure_steps", ctypes.c_int64), ("fallback_steps", ctypes.c_int64),
                ("last_residual", ctypes.c_float), ("moved_m3", ctypes.c_double)]


_SIGS = {
    "silt_conv3x3_forward": [_p, _p, _p, _p, _p, _p, _i, _i, _i, _i, _i, _i, _p],
    "silt_conv3x3_wgrad": [_p, _p, _p, _p, _i, _i, _i, _i, _i, _p],
    "silt_closure_loss_grad": [_p, _p, _p, _p, _p, _i, _i, _i, _f, _p],
    "silt_closure_step_loss_grad": [_p, _p, _p, _p, _f, _p, _p, _i, _f, _p],
    "silt_closure_adam": [_p, _p, _p, _p, _i, _f, _f, _f, _f, _i, _p],
    "silt_closure_pack": [_p, _p, _p, _i, _i, _p],
    "silt_closure_create": [_p, _i, _p, _i, ctypes.POINTER(_p)],
    "silt_closure_destroy": [_p],
    "silt_set_coupling": [_p, _i, _p, _f],
    "silt_closure_features": [_p, _p, _p, _p],
    "silt_get_closure_stats": [_p, ctypes.POINTER(ClosureStats)],
    "silt_closure_wait_status": [ctypes.POINTER(_i), _p],
    "silt_closure_wait_probe": [_i, _p],
}
_bound = {}


def fn(name):
    """The library entry point `name` with its argument types."""
    f = _bound.get(name)
    if f is None:
        f = getattr(silt_b200.lib(), name)
        f.argtypes = _SIGS[name]
        f.restype = ctypes.c_int
        _bound[name] = f
    return f


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def conv3x3(x, w_fwd, bias=None, gate=None, relu=False, cout=None, want_bf16=True, want_f32=False):
    """y = act(conv3x3(x, w) + bias) on the tensor cores. x: [n, h, w, cin]
    BF16; w_fwd: [cout, 9, cin] BF16. Returns (y_bf16 or None, y_f32 or None)."""
    import torch

    n, h, wd, cin = x.shape
    cout = cout or w_fwd.shape[0]
    y = torch.empty((n, h, wd, cout), dtype=torch.bfloat16, device=x.device) if want_bf16 else None
    y32 = torch.empty((n, h, wd, cout), dtype=torch.float32, device=x.device) if want_f32 else None
    silt_b200.check(fn("silt_conv3x3_forward")(_ptr(x), _ptr(w_fwd), _ptr(bias), _ptr(gate), _ptr(y), _ptr(y32),
                                               n, h, wd, cin, cout, int(relu), _stream()), "conv3x3_forward")
    return y, y32


def wgrad(x, dy, dw, db):
    """dw [9, cin, cout] += sum x[p + tap] dy[p]; db [cout] += sum dy (FP32)."""
    n, h, wd, cin = x.shape
    cout = dy.shape[-1]
    silt_b200.check(fn("silt_conv3x3_wgrad")(_ptr(x), _ptr(dy), _ptr(dw), _ptr(db), n, h, wd, cin, cout,
                                             _stream()), "conv3x3_wgrad")


def wait_status():
    """1 if a tensor-core kernel gave up a bounded wait since the last call (reads and clears)."""
    g = _i(0)
    silt_b200.check(fn("silt_closure_wait_status")(ctypes.byref(g), _stream()), "closure_wait_status")
    return g.value


def wait_probe(polls):
    """One CTA waits at most `polls` polls on an mbarrier phase nothing completes."""
    silt_b200.check(fn("silt_closure_wait_probe")(int(polls), _stream()), "closure_wait_probe")


def pack(w32, cin, cout, fwd=None, bwd=None):
    silt_b200.check(fn("silt_closure_pack")(_ptr(w32), _ptr(fwd), _ptr(bwd), cin, cout, _stream()), "closure_pack")


def split_params(p):
    """Views of the FP32 parameter vector: {"W1": [9, 16, 32], "b1": [32], ...}."""
    out, o = {}, 0
    for name, cin, cout in LAYERS:
        out["W" + name] = p[o:o + 9 * cin * cout].view(9, cin, cout)
        o += 9 * cin * cout
        out["b" + name] = p[o:o + cout]
        o += cout
    assert o == NPARAM
    return out


def init_params(seed=0):
    """He-initialised weights, zero biases; the last layer starts small so the
    untrained correction is near zero. Output channels >= OUT_USED stay 0."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, cin, cout in LAYERS:
        fan_in = 9 * (IN_USED if name == "1" else cin)
        w = rng.normal(0.0, np.sqrt(2.0 / fan_in), size=(9, cin, cout)).astype(np.float32)
        if name == "1":
            w[:, IN_USED:, :] = 0.0
        if name == "3":
            w *= 0.1
            w[:, :, OUT_USED:] = 0.0
        parts += [w.ravel(), np.zeros(cout, np.float32)]
    return np.concatenate(parts)


class Net:
    """The closure network on the device: FP32 master parameters, BF16
    packed weights for the forward and input-gradient convolutions."""

    def __init__(self, params=None, device="cuda"):
        import torch

        p = init_params() if params is None else np.asarray(params, np.float32)
        assert p.size == NPARAM
        self.p = torch.tensor(p, device=device)
        self.fwd = {n: torch.empty((co, 9, ci), dtype=torch.bfloat16, device=device) for n, ci, co in LAYERS}
        self.bwd = {n: torch.empty((ci, 9, co), dtype=torch.bfloat16, device=device) for n, ci, co in LAYERS}
        self.repack()

    def repack(self):
        P = split_params(self.p)
        for n, ci, co in LAYERS:
            pack(P["W" + n], ci, co, self.fwd[n], self.bwd[n])

    def forward(self, x):
        """x [n, h, w, 16] BF16 -> (a1, a2, y [n, h, w, 16] FP32)."""
        P = split_params(self.p)
        a1, _ = conv3x3(x, self.fwd["1"], P["b1"], relu=True)
        a2, _ = conv3x3(a1, self.fwd["2"], P["b2"], relu=True)
        _, y = conv3x3(a2, self.fwd["3"], P["b3"], want_bf16=False, want_f32=True)
        return a1, a2, y

    def grads(self, x, a1, a2, dy):
        """Parameter gradient (FP32, NPARAM) of the loss whose output gradient
        is dy [n, h, w, 16] BF16."""
        import torch

        g = torch.zeros(NPARAM, dtype=torch.float32, device=self.p.device)
        G = split_params(g)
        wgrad(a2, dy, G["W3"], G["b3"])
        dz2, _ = conv3x3(dy, self.bwd["3"], gate=a2, cout=HID)
        wgrad(a1, dz2, G["W2"], G["b2"])
        dz1, _ = conv3x3(dz2, self.bwd["2"], gate=a1, cout=HID)
        wgrad(x, dz1, G["W1"], G["b1"])
        # Padded input and output channels stay exactly zero.
        G["W1"][:, IN_USED:, :] = 0.0
        G["W3"][:, :, OUT_USED:] = 0.0
        G["b3"][OUT_USED:] = 0.0
        return g


def loss_grad(y, target, weight=None):
    """Weighted MSE of y[..., :4] against target [..., 4]; returns (dy BF16, loss tensor FP64)."""
    import torch

    n_pix = y.numel() // COUT
    dy = torch.empty(y.shape, dtype=torch.bfloat16, device=y.device)
    loss = torch.zeros(1, dtype=torch.float64, device=y.device)
    scale = 1.0 / float(n_pix * OUT_USED)
    silt_b200.check(fn("silt_closure_loss_grad")(_ptr(y), _ptr(target), _ptr(weight), _ptr(dy), _ptr(loss), n_pix,
                                                 COUT, OUT_USED, scale, _stream()), "closure_loss_grad")
    return dy, loss


def step_loss_grad(y, t, scale, inv_var, lam=0.0):
    """Loss of the step correction (mean over the crops' cells): the depth
    change the predicted transfers make and the predicted velocity change
    against t [n, 32, 32, 8] FP32 (water and slurry depth change in m; water
    u, v and slurry u, v change in m/s; water and slurry velocity weights),
    scale [8] and inv_var [6] FP32 device tensors. Returns (dy BF16, loss FP64)."""
    import torch

    n = y.shape[0]
    dy = torch.empty(y.shape, dtype=torch.bfloat16, device=y.device)
    loss = torch.zeros(1, dtype=torch.float64, device=y.device)
    norm = 1.0 / float(n * CROP * CROP)
    silt_b200.check(fn("silt_closure_step_loss_grad")(_ptr(y), _ptr(t), _ptr(scale), _ptr(inv_var), float(lam),
                                                      _ptr(dy), _ptr(loss), n, norm, _stream()),
                    "closure_step_loss_grad")
    return dy, loss


class Adam:
    def __init__(self, net, lr=2e-3, betas=(0.9, 0.999), eps=1e-8):
        import torch

        self.net, self.lr, self.b1, self.b2, self.eps = net, lr, betas[0], betas[1], eps
        self.m = torch.zeros_like(net.p)
        self.v = torch.zeros_like(net.p)
        self.t = 0

    def step(self, g, lr=None):
        self.t += 1
        silt_b200.check(fn("silt_closure_adam")(_ptr(self.net.p), _ptr(self.m), _ptr(self.v), _ptr(g), NPARAM,
                                                float(lr or self.lr), self.b1, self.b2, self.eps, self.t, _stream()),
                        "closure_adam")
        self.net.repack()


class Closure:
    """A trained network uploaded for the step (silt_closure_create)."""

    def __init__(self, params, norm, device=0):
        params = np.ascontiguousarray(params, np.float32)
        norm = np.ascontiguousarray(norm, np.float32)
        if params.size != NPARAM or norm.size != NNORM:
            raise ValueError("closure: parameter or normalisation size")
        h = ctypes.c_void_p()
        silt_b200.check(fn("silt_closure_create")(params.ctypes.data_as(_p), NPARAM, norm.ctypes.data_as(_p), device,
                                                  ctypes.byref(h)), "closure_create")
        self.h = h

    def close(self):
        if self.h:
            fn("silt_closure_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_coupling(sheet, mode, net=None, threshold=0.25):
    silt_b200.check(fn("silt_set_coupling")(sheet.h, int(mode), net.h if net is not None else None, float(threshold)),
                    "set_coupling")


def features(sheet, net, x):
    """The network input of the sheet's state and queued tires into x [1, 32, 32, 16] BF16; returns the crop's (i, j)."""
    origin = (ctypes.c_int32 * 2)()
    silt_b200.check(fn("silt_closure_features")(sheet.h, net.h, _ptr(x), origin), "closure_features")
    return int(origin[0]), int(origin[1])


def stats(sheet):
    s = ClosureStats()
    silt_b200.check(fn("silt_get_closure_stats")(sheet.h, ctypes.byref(s)), "closure_stats")
    return {k: getattr(s, k) for k, _ in ClosureStats._fields_}
