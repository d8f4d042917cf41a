"""The warm-start network on the GPU: its forward pass and gradients against
torch autograd on the same BF16 weights, and what the trained network gains
over the free-stream start (solver cycles to the same residual tolerance)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from finflo_b200 import warmstart as m
    return m


def _torch_reference(net, x, tgt):
    """The same network in torch FP32 autograd, rounding to BF16 where the
    kernels store BF16 (GEMM operands); returns the loss and the flat
    gradient in the layout of net.g."""
    import torch.nn.functional as F
    w = net.w.detach().clone().requires_grad_(True)
    bf = lambda t: t.to(torch.bfloat16).float()

    def b(l):
        return w[l.boff:l.boff + l.n]

    # straight-through BF16 rounding of the weights: the gradient w.r.t. the
    # rounded weight is the gradient w.r.t. the master weight
    def Wst(l):
        m = w[l.off:l.off + l.n * l.k].view(l.n, l.k)
        return m + (bf(m) - m).detach()

    def rnd(t):
        return t + (bf(t) - t).detach()

    h = rnd(x.float())
    for l in net.L[:4]:
        z = h @ Wst(l).T + b(l)
        h = rnd(F.silu(z) if l.act else z)
    a = h.reshape(-1, net.L[4].k)
    for l in net.L[4:-1]:
        z = a @ Wst(l).T + b(l)
        a = rnd(F.silu(z)).reshape(-1, net.L[4].k if l.name.startswith("up") else l.n)
    lo = net.L[-1]
    pred = a @ Wst(lo).T + b(lo)
    loss = ((pred[:, :tgt.shape[1]] - tgt) ** 2).mean()
    loss.backward()
    return loss.item(), w.grad


def test_forward_and_gradients_match_torch(ws):
    net = ws.WarmStartNet(seed=1)
    g = torch.Generator().manual_seed(2)
    x = torch.zeros(2, ws.IN_PAD)
    x[:, :2] = torch.rand(2, 2, generator=g) * 2 - 1
    x = x.cuda()
    tgt = torch.randn(2 * 65536, ws.NVAR, generator=g).cuda()
    net.forward(x)
    loss = net.backward(tgt).item()
    torch.cuda.synchronize()
    net.nn.error()
    ref_loss, ref_g = _torch_reference(net, x, tgt)
    assert abs(loss - ref_loss) <= 2e-3 * ref_loss
    # per layer: BF16 gradients of the activations -> a few per cent
    for l in net.L:
        a = net.g[l.off:l.off + l.n * l.k]
        r = ref_g[l.off:l.off + l.n * l.k]
        assert (a - r).norm().item() <= 5e-2 * r.norm().item() + 1e-12, l.name
        a, r = net.g[l.boff:l.boff + l.n], ref_g[l.boff:l.boff + l.n]
        assert (a - r).norm().item() <= 5e-2 * r.norm().item() + 1e-12, l.name + " bias"


def test_warm_start_beats_the_free_stream(ws):
    """What the trained network gains: trained on 16 solver solutions, its
    prediction as the start (with the FP32 implicit stage) reaches the
    tolerance -- 2 decades below the free-stream start's first-cycle density
    residual -- in fewer cycles in total over held-out cases than the plain
    FP64 solver from the free stream."""
    r = ws.run_config(ntrain=16, ntest=3, cycles=500, steps=1500, log=print)
    print("cycles to tolerance (free stream FP64, warm start FP32):",
          [(c["base_cycles"], c["warm_cycles"]) for c in r["cases"]])
    assert r["loss"][-1][1] < 0.7 * r["loss"][0][1]
    assert all(c["base_reached"] for c in r["cases"])
    assert all(c["warm_start_decades"] > 0.3 for c in r["cases"])   # the prediction starts closer
    assert r["warm_cycles"] < r["base_cycles"]
