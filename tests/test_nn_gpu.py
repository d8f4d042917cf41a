"""The warm-start network's tensor-core kernels against torch FP32 math on
the same BF16-rounded operands (GPU)."""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nn():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from finflo_b200 import nn as m
    m.lib()
    return m


def _bf(shape, seed, scale=1.0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return (torch.randn(*shape, generator=g) * scale).to(torch.bfloat16).cuda()


# (M, N, K): single tile, ragged M and N, N > 256 (two column tiles), K > 64
# (several staged K chunks, both smem stages reused), the decoder's shapes.
SHAPES = [(1, 16, 16), (200, 64, 32), (1000, 256, 32), (300, 512, 256), (130, 40, 48), (4096, 32, 32),
          (129, 16, 208)]


@pytest.mark.parametrize("M,N,K", SHAPES)
def test_gemm_matches_fp32(nn, M, N, K):
    A, B = _bf((M, K), 1), _bf((N, K), 2)
    bias = torch.randn(N, generator=torch.Generator().manual_seed(3)).cuda()
    zf = torch.full((M, N), float("nan"), device="cuda")
    yb = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
    nn.gemm(A, B, bias=bias, act=1, zf=zf, yb=yb)
    torch.cuda.synchronize()
    nn.error()
    ref = A.float() @ B.float().T + bias
    tol = 1e-5 * K ** 0.5 * ref.abs().max().item() + 1e-6
    assert (zf - ref).abs().max().item() <= tol
    ys = torch.nn.functional.silu(ref)
    assert (yb.float() - ys).abs().max().item() <= 1e-2 * ys.abs().max().item() + 1e-3


def test_gemm_split_k_atomic(nn):
    M, N, K = 32, 256, 4096
    A, B = _bf((M, K), 4), _bf((N, K), 5)
    zf = torch.zeros((M, N), device="cuda")
    nn.gemm(A, B, zf=zf, atomic=True, ksplit=512)
    torch.cuda.synchronize()
    nn.error()
    ref = A.float() @ B.float().T
    assert (zf - ref).abs().max().item() <= 1e-5 * K ** 0.5 * ref.abs().max().item()


def test_gemm_rejects_bad_shapes(nn):
    A, B = _bf((8, 24), 6), _bf((16, 24), 7)   # K not a multiple of 16
    zf = torch.zeros((8, 16), device="cuda")
    with pytest.raises(nn.NNError):
        nn.gemm(A, B, zf=zf)


def test_elementwise_kernels(nn):
    g = torch.Generator().manual_seed(8)
    z = torch.randn(1000, 48, generator=g).cuda()
    dy = torch.randn(1000, 48, generator=g).cuda()
    dzb = torch.empty(1000, 48, dtype=torch.bfloat16, device="cuda")
    dzf = torch.empty(1000, 48, device="cuda")
    nn.silu_bwd(dy, z, dzb, dzf)
    s = torch.sigmoid(z)
    ref = dy * s * (1 + z * (1 - s))
    assert (dzf - ref).abs().max().item() < 1e-5
    out = torch.zeros(48, device="cuda")
    nn.colsum(dzf, out)
    assert (out - ref.sum(0)).abs().max().item() < 1e-3
    x = _bf((100, 40), 9)
    t = torch.empty(40, 128, dtype=torch.bfloat16, device="cuda")
    nn.transpose(x, t, rows_pad=128)
    assert torch.equal(t[:, :100], x.T) and bool((t[:, 100:] == 0).all())
    pred = torch.randn(300, 16, generator=g).cuda()
    tgt = torch.randn(300, 5, generator=g).cuda()
    grad = torch.empty(300, 16, dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, device="cuda")
    nn.mse(pred, tgt, grad, loss)
    d = pred[:, :5] - tgt
    assert abs(loss.item() - (d ** 2).mean().item()) < 1e-4
    gref = 2 * d / d.numel()   # the gradient is stored in BF16 (8 significant bits)
    assert (grad[:, :5].float() - gref).abs().max().item() <= 4e-3 * gref.abs().max().item()
    assert bool((grad[:, 5:] == 0).all())


def test_adam_matches_torch(nn):
    g = torch.Generator().manual_seed(10)
    w0 = torch.randn(32, 24, generator=g)
    grads = [torch.randn(32, 24, generator=g) for _ in range(3)]
    w = w0.clone().cuda()
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    w16 = torch.empty(32, 24, dtype=torch.bfloat16, device="cuda")
    w16t = torch.empty(24, 32, dtype=torch.bfloat16, device="cuda")
    p = w0.clone().requires_grad_(True)
    opt = torch.optim.Adam([p], lr=1e-2)
    for i, gr in enumerate(grads):
        nn.adam(w, gr.cuda(), m, v, i + 1, 1e-2, w16=w16, w16t=w16t, rows=32)
        p.grad = gr.clone()
        opt.step()
    torch.cuda.synchronize()
    assert (w.cpu() - p.detach()).abs().max().item() < 1e-5
    assert torch.equal(w16t.T.contiguous(), w16)
