"""Tensor-core MLP kernels (forward and training gradients) against a torch FP32 reference with the
kernel's BF16 rounding points, and against the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _bf16(t):
    import torch

    return t.to(torch.bfloat16).to(torch.float32)


ACTS = {"gelu": L.ARC_MLP_ACT_GELU, "relu": L.ARC_MLP_ACT_RELU}


def _torch_forward(p, x, act="gelu"):
    """FP32 reference of the kernels' inference.  GELU: the activation's constants folded into the
    parameters as the library's weight image holds them (s W1, W2 / 2, W3 / 2 in BF16, s b in FP32,
    w4 / (2 s)), the folded activation z + z tanh(z).  ReLU: the parameters as stored, W in BF16.
    Both: BF16 inputs and hidden activations."""
    import torch

    P = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in M.unpack(p).items()}
    if act == "relu":
        h = _bf16(x)
        h1 = _bf16(torch.relu(h @ _bf16(P["W1"]).T + P["b1"]))
        h2 = _bf16(torch.relu(h1 @ _bf16(P["W2"]).T + P["b2"]))
        return torch.relu(h2 @ _bf16(P["W3"]).T + P["b3"]) @ P["w4"] + P["b4"][0]
    s = torch.tensor(0.851, dtype=torch.float32)
    g = lambda z: z + z * torch.tanh(z)  # noqa: E731
    h = _bf16(x)
    z1 = h @ _bf16(s * P["W1"]).T + s * P["b1"]
    h1 = _bf16(g(z1))
    z2 = h1 @ _bf16(0.5 * P["W2"]).T + s * P["b2"]
    h2 = _bf16(g(z2))
    z3 = h2 @ _bf16(0.5 * P["W3"]).T + s * P["b3"]
    h3 = g(z3)
    return h3 @ ((torch.tensor(0.5, dtype=torch.float32) / s) * P["w4"]) + P["b4"][0]


@pytest.fixture(scope="module")
def mlp(ctx):
    h = C.c_void_p()
    L.check(ctx.lib.arc_mlp_create(ctx.handle, 7, C.byref(h)), "arc_mlp_create")
    yield h
    ctx.lib.arc_mlp_destroy(h)


def _params(ctx, h):
    p = np.zeros(M.NUM_PARAMS, np.float32)
    L.check(ctx.lib.arc_mlp_get_params(h, p.ctypes.data_as(C.POINTER(C.c_float)), M.NUM_PARAMS), "get")
    return p


@pytest.mark.parametrize("act", ["gelu", "relu"])
@pytest.mark.parametrize("rows", [1, 127, 128, 1000, 70000])
def test_forward_matches_torch_and_oracle(ctx, mlp, rows, act):
    import torch

    L.check(ctx.lib.arc_mlp_set_activation(mlp, ACTS[act]), "set_activation")
    assert ctx.lib.arc_mlp_get_activation(mlp) == ACTS[act]
    g = torch.Generator(device="cuda").manual_seed(rows)
    x = torch.randn(rows, 16, device="cuda", generator=g).to(torch.bfloat16).contiguous()
    out = torch.empty(rows, device="cuda")
    L.check(ctx.lib.arc_mlp_forward(mlp, C.c_void_p(x.data_ptr()), rows, C.c_void_p(out.data_ptr())), "forward")
    assert ctx.synchronize() == 0
    L.check(ctx.lib.arc_mlp_set_activation(mlp, L.ARC_MLP_ACT_GELU), "set_activation")
    p = _params(ctx, mlp)
    ref = _torch_forward(p, x.float(), act)
    err = (out - ref).abs().max().item()
    assert err <= 2e-3 * max(1.0, ref.abs().max().item()), err
    if rows <= 1000:
        y64, _ = M.forward(p.astype(np.float64), x.float().cpu().numpy(), act)
        assert np.max(np.abs(out.cpu().numpy() - y64)) <= 3e-2 * max(1.0, np.abs(y64).max())
        yb = M.forward_bf16(p, x.float().cpu().numpy(), act)
        assert np.max(np.abs(out.cpu().numpy() - yb)) <= 2e-3 * max(1.0, np.abs(yb).max())


@pytest.mark.parametrize("act", ["gelu", "relu"])
@pytest.mark.parametrize("loss", ["bce", "squared"])
def test_gradients_match_torch_and_oracle(ctx, mlp, loss, act):
    import torch

    rows = 1000
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn(rows, 16, device="cuda", generator=g).to(torch.bfloat16).contiguous()
    if loss == "bce":
        lab = (torch.rand(rows, device="cuda", generator=g) > 0.5).float()
    else:
        lab = torch.randn(rows, device="cuda", generator=g) * 0.5
    wts = torch.rand(rows, device="cuda", generator=g) + 0.5
    kind = L.ARC_MLP_LOSS_BCE if loss == "bce" else L.ARC_MLP_LOSS_SQUARED
    L.check(ctx.lib.arc_mlp_set_loss(mlp, kind), "set_loss")
    L.check(ctx.lib.arc_mlp_set_activation(mlp, ACTS[act]), "set_activation")
    assert ctx.lib.arc_mlp_get_loss(mlp) == kind
    grads = np.zeros(M.NUM_PARAMS, np.float32)
    loss_v = C.c_float()
    L.check(ctx.lib.arc_mlp_gradients(mlp, C.c_void_p(x.data_ptr()), C.c_void_p(lab.data_ptr()),
                                      C.c_void_p(wts.data_ptr()), rows, float(wts.sum().item()),
                                      grads.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss_v)), "gradients")
    p = _params(ctx, mlp)
    L.check(ctx.lib.arc_mlp_set_loss(mlp, L.ARC_MLP_LOSS_BCE), "set_loss")
    L.check(ctx.lib.arc_mlp_set_activation(mlp, L.ARC_MLP_ACT_GELU), "set_activation")
    l64, g64 = M.loss_and_grad(p.astype(np.float64), x.float().cpu().numpy(), lab.cpu().numpy(), wts.cpu().numpy(),
                               loss=loss, act=act)
    assert abs(loss_v.value - l64) <= 1e-2 * abs(l64)
    # torch autograd with the kernel's rounding points (straight-through in the backward)
    P = {k: torch.tensor(v, dtype=torch.float32, device="cuda", requires_grad=True) for k, v in M.unpack(p).items()}
    if act == "relu":
        f = torch.relu
    else:
        f = lambda z: 0.5 * z * (1 + torch.tanh(0.851 * z))  # noqa: E731  (x sigma(1.702 x))
    st = lambda t: t + (_bf16(t) - t).detach()  # noqa: E731
    z1 = st(x.float()) @ st(P["W1"]).T + P["b1"]
    h1 = st(f(z1))
    z2 = h1 @ st(P["W2"]).T + P["b2"]
    h2 = st(f(z2))
    z3 = h2 @ st(P["W3"]).T + P["b3"]
    y = f(z3) @ P["w4"] + P["b4"][0]
    if loss == "bce":
        per = torch.nn.functional.binary_cross_entropy_with_logits(y, lab, reduction="none")
    else:
        per = (y - lab) ** 2
    ref_loss = (wts * per).sum() / wts.sum()
    ref_loss.backward()
    gt = np.concatenate([P[k].grad.detach().cpu().numpy().ravel() for k, _ in M.SIZES])
    for ref, tol in ((gt, 0.03), (g64, 0.05)):
        rel = np.linalg.norm(grads - ref) / np.linalg.norm(ref)
        assert rel < tol, rel
        cos = grads @ ref / (np.linalg.norm(grads) * np.linalg.norm(ref))
        assert cos > 0.998


@pytest.mark.parametrize("act", ["gelu", "relu"])
def test_training_learns_a_separable_rule(ctx, act):
    import torch

    h = C.c_void_p()
    L.check(ctx.lib.arc_mlp_create(ctx.handle, 1, C.byref(h)), "create")
    L.check(ctx.lib.arc_mlp_set_activation(h, ACTS[act]), "set_activation")
    g = torch.Generator(device="cuda").manual_seed(5)
    n = 65536
    x = torch.randn(n, 16, device="cuda", generator=g)
    lab = ((x[:, 0] + 0.5 * x[:, 1] - 0.25 * x[:, 2]) > 0.1).float()
    xb = x.to(torch.bfloat16).contiguous()
    losses = []
    for step in range(300):
        i = (step * 4096) % n
        acc = torch.zeros(1, device="cuda")
        L.check(ctx.lib.arc_mlp_train_step(h, C.c_void_p(xb[i:i + 4096].data_ptr()), C.c_void_p(lab[i:i + 4096].data_ptr()),
                                           None, 4096, 4096.0, 3e-3, C.c_void_p(acc.data_ptr())), "train")
        losses.append(acc)
    out = torch.empty(n, device="cuda")
    L.check(ctx.lib.arc_mlp_forward(h, C.c_void_p(xb.data_ptr()), n, C.c_void_p(out.data_ptr())), "forward")
    assert ctx.synchronize() == 0
    acc = ((out > 0).float() == lab).float().mean().item()
    first = sum(l.item() for l in losses[:10]) / 10
    last = sum(l.item() for l in losses[-10:]) / 10
    ctx.lib.arc_mlp_destroy(h)
    assert last < 0.3 * first and acc > 0.97, (first, last, acc)
