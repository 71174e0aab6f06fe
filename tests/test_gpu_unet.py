"""The learned-guess network's CUDA forward and backward against a torch-CPU FP32
reference that rounds weights and activations to BF16 at the same points (gradients
flow straight through the rounding), on a grid with odd sizes at every level."""
import pytest
import torch
import torch.nn.functional as F

from meltpooldg_b200 import learned as LG

pytestmark = pytest.mark.gpu


def bf(t):
    return t + (t.to(torch.bfloat16).float() - t).detach()


def pool(t):
    nz, ny, nx = t.shape[-3:]
    pz, py, px = nz % 2, ny % 2, nx % 2
    tp = F.pad(t, (0, px, 0, py, 0, pz))
    ones = F.pad(torch.ones_like(t[:, :1]), (0, px, 0, py, 0, pz))
    return F.avg_pool3d(tp, 2) / F.avg_pool3d(ones, 2)


def up(t, shape):
    for d, n in zip((2, 3, 4), shape):
        t = t.repeat_interleave(2, dim=d).narrow(d, 0, n)
    return t


class ConvBF16Backward(torch.autograd.Function):
    """conv3d whose input gradient is formed from the output gradient rounded to BF16 (as the
    tensor-core data gradient does) and whose weight and bias gradients from the FP32 one."""

    @staticmethod
    def forward(ctx, t, w, b):
        ctx.save_for_backward(t, w)
        return F.conv3d(t, w, b, padding=1)

    @staticmethod
    def backward(ctx, g):
        t, w = ctx.saved_tensors
        gi = torch.nn.grad.conv3d_input(t.shape, w, g.to(torch.bfloat16).float(), padding=1)
        gw = torch.nn.grad.conv3d_weight(t, w.shape, g, padding=1)
        return gi, gw, g.sum(dim=(0, 2, 3, 4))


def reference(params, x, dims, bf16_dgrad=True):
    nx, ny, nz = dims
    layers = LG.unpack(params)

    def conv(t, l, relu=True, add=None):
        w, b = layers[l]
        if bf16_dgrad:
            r = ConvBF16Backward.apply(t, bf(w), b)
        else:
            r = F.conv3d(t, bf(w), b, padding=1)
        if add is not None:
            r = r + add
        return bf(torch.relu(r)) if relu else r

    x0 = bf(x.view(1, 3, nz, ny, nx))
    e0 = conv(conv(x0, 0), 1)
    e1 = conv(conv(bf(pool(e0)), 2), 3)
    e2 = conv(conv(bf(pool(e1)), 4), 5)
    e3 = conv(conv(bf(pool(e2)), 6), 7)
    d2 = conv(conv(up(e3, e2.shape[-3:]), 8, add=e2), 9)
    d1 = conv(conv(up(d2, e1.shape[-3:]), 10, add=e1), 11)
    d0 = conv(conv(up(d1, e0.shape[-3:]), 12, add=e0), 13)
    return conv(d0, 14, relu=False).reshape(-1)


@pytest.mark.parametrize("tc_bwd", [True, False])
def test_forward_and_parameter_gradients_match_torch_reference(tc_bwd, monkeypatch):
    """Default: the data gradients on the tensor cores (the output gradient rounded to BF16
    before each one, as the reference here does too); MPDG_UNET_TC_BWD=0: on the CUDA cores in
    FP32."""
    monkeypatch.setenv("MPDG_UNET_TC_BWD", "1" if tc_bwd else "0")
    dims = (19, 14, 11)  # odd/even mixes: 19->10->5->3, 14->7->4->2, 11->6->3->2
    net = LG.UNet(dims, seed=3)
    g = torch.Generator().manual_seed(0)
    n = dims[0] * dims[1] * dims[2]
    x = torch.randn(3 * n, generator=g)
    y = net.forward(x.cuda()).cpu()
    p = net.get_params().cpu().requires_grad_(True)
    y_ref = reference(p, x, dims, bf16_dgrad=tc_bwd)
    err = (y - y_ref.detach()).norm() / y_ref.detach().norm()
    assert err < 2e-2, err
    gy = torch.randn(n, generator=g)
    grad = net.backward(gy.cuda()).cpu()
    (y_ref * gy).sum().backward()
    gr = p.grad
    cos = torch.dot(grad, gr) / (grad.norm() * gr.norm())
    assert cos > 0.999, cos
    assert (grad - gr).norm() / gr.norm() < 5e-2
    # every layer's weights receive a gradient of the right size
    for (gw, _), (rw, _) in zip(LG.unpack(grad), LG.unpack(gr)):
        assert torch.allclose(gw.norm(), rw.norm(), rtol=0.1)


def test_training_reduces_the_loss():
    dims = (17, 17, 17)
    net = LG.UNet(dims, seed=5)
    g = torch.Generator().manual_seed(1)
    n = 17 ** 3
    x = torch.randn(3 * n, generator=g).cuda()
    t = (0.5 * x.view(3, n)[0] - 0.25 * x.view(3, n)[1]).contiguous()
    first = net.train_step(x, t, 1e-3)
    for _ in range(150):
        last = net.train_step(x, t, 1e-3)
    assert last < 0.2 * first, (first, last)


def test_tensor_core_forward_matches_cuda_core_forward(monkeypatch):
    """The tcgen05 implicit-GEMM convolutions against the CUDA-core ones (same BF16
    weights and activations, FP32 accumulation in both) on a grid whose x and y sizes
    leave partial 8 x 16 tiles at every level."""
    dims = (40, 33, 9)
    n = dims[0] * dims[1] * dims[2]
    monkeypatch.delenv("MPDG_UNET_TC", raising=False)
    net_tc = LG.UNet(dims, seed=7)
    monkeypatch.setenv("MPDG_UNET_TC", "0")
    net_cc = LG.UNet(dims, seed=7)
    g = torch.Generator().manual_seed(2)
    for _ in range(2):
        x = torch.randn(3 * n, generator=g).cuda()
        y_tc, y_cc = net_tc.forward(x), net_cc.forward(x)
        err = (y_tc - y_cc).norm() / y_cc.norm()
        assert err < 1e-2, err
        # after an update of the weights the packed copy follows
        p = net_cc.get_params()
        p.add_(0.01 * torch.randn(p.numel(), generator=g).cuda())
        net_tc.set_params(p)
        net_cc.set_params(p)


def test_tensor_core_backward_matches_cuda_core_backward(monkeypatch):
    """Parameter gradients with the data gradients on the tensor cores against the FP32
    CUDA-core ones, same forward, on a grid with partial tiles at every level."""
    dims = (40, 33, 9)
    n = dims[0] * dims[1] * dims[2]
    monkeypatch.setenv("MPDG_UNET_TC_BWD", "1")
    net_tc = LG.UNet(dims, seed=11)
    monkeypatch.setenv("MPDG_UNET_TC_BWD", "0")
    net_cc = LG.UNet(dims, seed=11)
    g = torch.Generator().manual_seed(4)
    x = torch.randn(3 * n, generator=g).cuda()
    gy = torch.randn(n, generator=g).cuda()
    net_tc.forward(x)
    net_cc.forward(x)
    a, b = net_tc.backward(gy), net_cc.backward(gy)
    cos = torch.dot(a, b) / (a.norm() * b.norm())
    assert cos > 0.9999, cos
    assert (a - b).norm() / b.norm() < 2e-2
