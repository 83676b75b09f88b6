"""The tensor-core GEMM (tcgen05, BF16 in, FP32 accumulate) and the MLP's
forward/backward/Adam kernels against torch FP32 products and the float64 CPU
oracle (oracle/mlp_oracle.py).

Tolerances: GEMM outputs to 1e-5 relative to the magnitude of the FP32
reference (only summation order differs); MLP forward to 1e-2 relative
(activations are stored as BF16 between layers); gradients to 3e-2 relative
Frobenius error per layer (BF16 deltas)."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as MO
from rlmusclev2_b200 import _capi as capi
from rlmusclev2_b200.cagenet import DIMS, CageMLP, gemm

pytestmark = pytest.mark.gpu


def _lib():
    return capi.load()


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (300, 256, 256), (1000, 48, 128), (3, 256, 1280), (129, 16, 64)])
def test_gemm_matches_fp32_product(m, n, k):
    torch.manual_seed(m + n + k)
    dev = torch.device("cuda:0")
    a = torch.randn(m, k, device=dev).to(torch.bfloat16)
    b = torch.randn(n, k, device=dev).to(torch.bfloat16)
    ref = a.float() @ b.float().t()
    out = torch.full((m, n), float("nan"), device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream()
    import ctypes as C
    gemm(_lib(), C.c_void_p(s.cuda_stream), a, b, m, n, k, out_f32=out, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    err = (out - ref).abs().max().item() / ref.abs().max().item()
    print(f"gemm {m}x{n}x{k}: rel err {err:.2e}")
    assert err < 1e-5


def test_gemm_epilogues():
    import ctypes as C
    torch.manual_seed(1)
    dev = torch.device("cuda:0")
    m, n, k = 260, 256, 128
    a = torch.randn(m, k, device=dev).to(torch.bfloat16)
    b = (0.1 * torch.randn(n, k, device=dev)).to(torch.bfloat16)
    bias = torch.randn(n, device=dev)
    g = torch.randn(m, n, device=dev)
    pre = torch.zeros(m, n, device=dev)
    hb = torch.zeros(m, n, dtype=torch.bfloat16, device=dev)
    ht = torch.zeros(n, 384, dtype=torch.bfloat16, device=dev)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    gemm(_lib(), s, a, b, m, n, k, bias=bias, act=1, gelu_grad_of=g, out_pre=pre, out_bf16=hb, out_bf16_t=ht)
    torch.cuda.synchronize()
    z = (a.double() @ b.double().t() + bias.double()).cpu().numpy() * MO.gelu_grad(g.double().cpu().numpy())
    np.testing.assert_allclose(pre.cpu().numpy(), z, rtol=1e-4, atol=1e-4)
    y = MO.gelu(pre.double().cpu().numpy())
    np.testing.assert_allclose(hb.float().cpu().numpy(), y, rtol=1e-2, atol=1e-2)
    np.testing.assert_array_equal(ht[:, :m].t().float().cpu().numpy(), hb.float().cpu().numpy())


def _oracle_weights(net):
    Ws = [MO.bf16_round(net.W[l].cpu().numpy()) for l in range(5)]
    bs = [net.b[l].double().cpu().numpy() for l in range(5)]
    return Ws, bs


def test_mlp_forward_backward_vs_oracle():
    torch.manual_seed(2)
    dev = torch.device("cuda:0")
    m = 777
    net = CageMLP(dev, m, seed=3)
    with torch.cuda.stream(net.stream):
        for l in range(5):
            net.b[l].copy_(0.1 * torch.randn(DIMS[l + 1], device=dev))
    net.refresh_copies()
    x = torch.randn(m, 64, device=dev).to(torch.bfloat16)
    tgt = torch.randn(m, 3, device=dev)
    with torch.cuda.stream(net.stream):
        net.X[:m].copy_(x)
        net.Xt[:, :m].copy_(x.t())
        net.loss.zero_()
    y = net.forward(m).clone()
    net.backward(m, tgt)
    torch.cuda.synchronize()
    assert int(net.status.item()) == 0
    Ws, bs = _oracle_weights(net)
    X = x.double().cpu().numpy()
    loss, Y, gW, gb = MO.loss_and_grads(X, Ws, bs, tgt.double().cpu().numpy())
    fe = np.abs(y.cpu().numpy() - Y).max() / np.abs(Y).max()
    gl = float(net.loss.item()) / (m * 3)
    print(f"forward rel err {fe:.2e}, loss gpu {gl:.5f} oracle {loss:.5f}")
    assert fe < 1e-2 and abs(gl - loss) / loss < 1e-2
    for l in range(5):
        gw = net.gW[l].double().cpu().numpy()
        e = np.linalg.norm(gw - gW[l]) / np.linalg.norm(gW[l])
        eb = np.linalg.norm(net.gb[l].double().cpu().numpy() - gb[l]) / np.linalg.norm(gb[l])
        print(f"layer {l}: dW rel err {e:.2e}, db rel err {eb:.2e}")
        assert e < 3e-2 and eb < 3e-2


def test_adam_training_reduces_loss():
    """A few hundred Adam steps on a fixed synthetic regression lower the loss."""
    torch.manual_seed(4)
    dev = torch.device("cuda:0")
    m = 1024
    net = CageMLP(dev, m, seed=5)
    x = torch.randn(m, 64, device=dev)
    tgt = torch.stack([torch.sin(x[:, 0]) + 0.5 * x[:, 1], x[:, 2] * x[:, 3], torch.tanh(x[:, 4])], 1)
    with torch.cuda.stream(net.stream):
        net.X[:m].copy_(x.to(torch.bfloat16))
        net.Xt[:, :m].copy_(x.t().to(torch.bfloat16))
    losses = []
    for it in range(300):
        with torch.cuda.stream(net.stream):
            net.loss.zero_()
        net.forward(m)
        net.backward(m, tgt)
        net.adam_step(lr=1e-3)
        if it in (0, 299):
            torch.cuda.synchronize()
            losses.append(float(net.loss.item()) / (m * 3))
    print("loss", losses)
    assert int(net.status.item()) == 0
    assert losses[1] < 0.2 * losses[0]


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (9472, 256, 256), (1000, 48, 128), (300, 16, 1280)])
def test_gemm_tma_operands_equal_thread_staged(m, n, k):
    """The TMA-fed kernel runs the same MMAs in the same k order as the
    thread-staged one: bit-identical outputs, including the zero-filled rows
    beyond m and n."""
    import ctypes as C
    torch.manual_seed(7 + m)
    dev = torch.device("cuda:0")
    a = torch.randn(m, k, device=dev).to(torch.bfloat16)
    b = torch.randn(n, k, device=dev).to(torch.bfloat16)
    bias = torch.randn(n, device=dev)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    outs = []
    for flags in (0, 1):
        out = torch.full((m, n), float("nan"), device=dev)
        hb = torch.zeros(m, n, dtype=torch.bfloat16, device=dev)
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        gemm(_lib(), s, a, b, m, n, k, bias=bias, act=1, out_f32=out, out_bf16=hb, status=st, flags=flags)
        torch.cuda.synchronize()
        assert int(st.item()) == 0
        outs.append((out, hb))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    ref = a.float() @ b.float().t() + bias
    y = outs[0][0]
    assert torch.isfinite(y).all()
    gl = 0.5 * ref * (1 + torch.tanh(0.7978845608028654 * (ref + 0.044715 * ref ** 3)))
    assert ((y - gl).abs().max() / gl.abs().max()).item() < 1e-4
