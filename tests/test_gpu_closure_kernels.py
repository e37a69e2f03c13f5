"""The closure's tensor-core kernels (tcgen05 implicit-GEMM 3x3 convolutions,
their input and weight gradients, the loss gradient, Adam, packing) against a
plain PyTorch FP32 reference of the same ops on the same BF16-rounded
operands. Both sides accumulate in FP32, so the FP32 outputs agree to
summation-order rounding (tolerance 1e-4 relative to the output scale);
BF16 outputs within one BF16 rounding (2^-8 relative)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import silt_closure as C

pytestmark = pytest.mark.gpu

TAPS = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def ref_conv(x, w_tcc, bias=None):
    """x [n, h, w, cin] FP32, w [9, cin, cout] -> [n, h, w, cout] FP32 (zero padding)."""
    k = w_tcc.view(3, 3, w_tcc.shape[1], w_tcc.shape[2]).permute(3, 2, 0, 1).contiguous()  # [cout, cin, 3, 3]
    y = torch.nn.functional.conv2d(x.permute(0, 3, 1, 2), k, bias=bias, padding=1)
    return y.permute(0, 2, 3, 1).contiguous()


def rand_bf16(shape, scale=1.0, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return (torch.randn(shape, device="cuda", generator=g) * scale).to(torch.bfloat16)


def close(a, b, rel):
    scale = float(b.abs().max()) + 1e-12
    return float((a - b).abs().max()) <= rel * scale, float((a - b).abs().max()) / scale


@pytest.mark.parametrize("cin,cout,h,w", [(16, 32, 32, 32), (32, 32, 19, 45), (32, 16, 200, 200)])
def test_conv_forward_matches_fp32_reference(cin, cout, h, w):
    n = 3
    x = rand_bf16((n, h, w, cin), seed=1)
    w32 = (rand_bf16((9, cin, cout), 0.2, seed=2)).float()
    b = torch.randn(cout, device="cuda") * 0.1
    fwd = torch.empty((cout, 9, cin), dtype=torch.bfloat16, device="cuda")
    C.pack(w32.contiguous(), cin, cout, fwd=fwd)
    y, y32 = C.conv3x3(x, fwd, b, relu=False, want_bf16=True, want_f32=True)
    ref = ref_conv(x.float(), w32, b)
    ok, err = close(y32, ref, 1e-4)
    assert ok, err
    ok, err = close(y.float(), ref, 2.0 ** -7)
    assert ok, err
    yr, _ = C.conv3x3(x, fwd, b, relu=True)
    ok, err = close(yr.float(), torch.relu(ref), 2.0 ** -7)
    assert ok, err


def test_conv_input_gradient_with_gate():
    n, h, w, cin, cout = 2, 32, 32, 32, 32
    x = rand_bf16((n, h, w, cin), seed=3)
    w32 = rand_bf16((9, cin, cout), 0.2, seed=4).float().contiguous()
    dy = rand_bf16((n, h, w, cout), seed=5)
    gate = rand_bf16((n, h, w, cin), seed=6)
    bwd = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device="cuda")
    C.pack(w32, cin, cout, bwd=bwd)
    _, dx32 = C.conv3x3(dy, bwd, gate=gate, cout=cin, want_bf16=False, want_f32=True)
    xr = x.float().requires_grad_(True)
    y = ref_conv(xr, w32)
    y.backward(dy.float())
    ref = xr.grad * (gate.float() > 0)
    ok, err = close(dx32, ref, 1e-4)
    assert ok, err


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16)])
def test_weight_gradient_matches_fp32_reference(cin, cout):
    n, h, w = 4, 32, 32
    x = rand_bf16((n, h, w, cin), seed=7)
    dy = rand_bf16((n, h, w, cout), seed=8)
    dw = torch.zeros((9, cin, cout), device="cuda")
    db = torch.zeros(cout, device="cuda")
    C.wgrad(x, dy, dw, db)
    wr = torch.zeros((9, cin, cout), device="cuda", requires_grad=True)
    br = torch.zeros(cout, device="cuda", requires_grad=True)
    y = ref_conv(x.float(), wr, br)
    y.backward(dy.float())
    ok, err = close(dw, wr.grad, 1e-4)
    assert ok, err
    ok, err = close(db, br.grad, 1e-4)
    assert ok, err


def test_loss_gradient_and_network_gradient_against_autograd():
    net = C.Net(C.init_params(seed=3))
    n = 2
    x = torch.zeros((n, 32, 32, C.CIN), dtype=torch.bfloat16, device="cuda")
    x[..., :C.IN_USED] = rand_bf16((n, 32, 32, C.IN_USED), seed=9)
    t = torch.randn((n, 32, 32, C.OUT_USED), device="cuda") * 0.1
    a1, a2, y = net.forward(x)
    dy, loss = C.loss_grad(y, t)
    ref_loss = ((y[..., :C.OUT_USED] - t) ** 2).mean()
    assert abs(float(loss) - float(ref_loss)) <= 1e-5 * float(ref_loss)
    g = net.grads(x, a1, a2, dy)
    # The same network in FP32 autograd with BF16-rounded weights and activations.
    P = {k: v.detach().clone().to(torch.bfloat16).float().requires_grad_(True) for k, v in C.split_params(net.p).items()}
    for k in ("b1", "b2", "b3"):
        P[k] = C.split_params(net.p)[k].detach().clone().requires_grad_(True)
    h1 = torch.relu(ref_conv(x.float(), P["W1"], P["b1"]))
    h2 = torch.relu(ref_conv(h1.to(torch.bfloat16).float(), P["W2"], P["b2"]))
    yr = ref_conv(h2.to(torch.bfloat16).float(), P["W3"], P["b3"])
    lr = ((yr[..., :C.OUT_USED] - t) ** 2).mean()
    lr.backward()
    G = C.split_params(g)
    for k in ("W3", "b3", "W2", "b2", "W1", "b1"):
        ref = P[k].grad.clone()
        if k == "W1":
            ref[:, C.IN_USED:, :] = 0
        if k == "W3":
            ref[:, :, C.OUT_USED:] = 0
        if k == "b3":
            ref[C.OUT_USED:] = 0
        ok, err = close(G[k], ref, 0.03)  # BF16 gradients through two ReLU layers
        assert ok, (k, err)


def test_adam_training_reduces_the_loss():
    net = C.Net(C.init_params(seed=5))
    opt = C.Adam(net, lr=3e-3)
    n = 16
    x = torch.zeros((n, 32, 32, C.CIN), dtype=torch.bfloat16, device="cuda")
    x[..., :C.IN_USED] = rand_bf16((n, 32, 32, C.IN_USED), seed=11)
    # A target the network can represent: a fixed random 3x3 map of the inputs.
    wt = torch.randn((9, C.IN_USED, C.OUT_USED), device="cuda") * 0.2
    t = ref_conv(x[..., :C.IN_USED].float(), wt).contiguous()
    first = None
    for it in range(150):
        a1, a2, y = net.forward(x)
        dy, loss = C.loss_grad(y, t)
        g = net.grads(x, a1, a2, dy)
        opt.step(g)
        if first is None:
            first = float(loss)
    a1, a2, y = net.forward(x)
    _, loss = C.loss_grad(y, t)
    assert float(loss) < 0.2 * first, (first, float(loss))
    p = C.split_params(net.p)
    assert float(p["W1"][:, C.IN_USED:, :].abs().max()) == 0.0
    assert float(p["W3"][:, :, C.OUT_USED:].abs().max()) == 0.0


def test_bounded_wait_gives_up_and_reports_without_a_fault():
    """The tensor-core kernels wait on mbarrier phases with a poll limit. A
    probe waits on a phase nothing completes, with a tiny limit: it must give
    up, the status must come back to the host (and clear on reading), and the
    context must stay usable: a convolution afterwards still matches the
    FP32 reference and reports no give-up."""
    assert C.wait_status() == 0
    C.wait_probe(1000)
    torch.cuda.synchronize()
    assert C.wait_status() == 1
    assert C.wait_status() == 0
    x = rand_bf16((2, 16, 16, 16), seed=5)
    w32 = rand_bf16((9, 16, 32), 0.2, seed=6).float()
    wf = torch.empty((32, 9, 16), dtype=torch.bfloat16, device="cuda")
    C.pack(w32.contiguous(), 16, 32, fwd=wf)
    _, y32 = C.conv3x3(x, wf, want_bf16=False, want_f32=True)
    ok, err = close(y32, ref_conv(x.float(), w32), 1e-4)
    assert ok, err
    assert C.wait_status() == 0
