"""GPU tests of the warm-start MLP: the tcgen05 BF16 product against a torch
FP32 product of the same BF16 operands, forward / loss / gradients against the
CPU oracle, one AdamW step against the oracle, training progress and
determinism."""
import numpy as np
import pytest

import tlfea_b200 as T
from oracle import mlp_oracle as MO

from .helpers import rel

pytestmark = pytest.mark.gpu

DIMS = [6, 256, 256, 256, 64]


@pytest.mark.parametrize("M,N,K", [(128, 256, 256), (256, 64, 16), (300, 272, 80), (512, 256, 512), (128, 16, 16),
                                   (1000, 528, 1040), (200, 48, 2048), (2048, 2048, 384), (4096, 1296, 320)])
def test_gemm_bf16_matches_fp32_product_of_bf16_operands(M, N, K):
    import torch

    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).cuda()
    D = torch.zeros(M, N, device="cuda")
    torch.cuda.synchronize()
    T.gemm_bf16(M, N, K, A.data_ptr(), K, B.data_ptr(), K, bias.data_ptr(), D.data_ptr(), N)
    ref = A.double() @ B.double().T + bias.double()
    # FP32 accumulation over K products inside the tensor core: the error bound
    # grows linearly with K (measured 1.0e-6 at K = 1040, 2.1e-6 at K = 2048)
    tol = 1e-6 * max(1.0, K / 512)
    assert rel(D.cpu().numpy(), ref.cpu().numpy()) < tol
    D2 = torch.zeros(M, N, device="cuda")
    torch.cuda.synchronize()
    T.gemm_bf16(M, N, K, A.data_ptr(), K, B.data_ptr(), K, 0, D2.data_ptr(), N)
    assert rel(D2.cpu().numpy(), (A.double() @ B.double().T).cpu().numpy()) < tol


def test_gemm_bf16_async_matches_the_synchronous_call():
    """The enqueue-only entry point gives the same product, bit for bit, and leaves
    the error flag at zero; grouped tile order is exercised by a grid of several
    row groups (M = 4480: 35 row tiles, groups of 16, 16 and 3)."""
    import torch

    M, N, K = 4480, 384, 256
    g = torch.Generator(device="cpu").manual_seed(7)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    D1 = torch.zeros(M, N, device="cuda")
    D2 = torch.zeros(M, N, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    T.gemm_bf16(M, N, K, A.data_ptr(), K, B.data_ptr(), K, 0, D1.data_ptr(), N)
    st = torch.cuda.current_stream()
    T.gemm_bf16_async(M, N, K, A.data_ptr(), K, B.data_ptr(), K, 0, D2.data_ptr(), N, flag.data_ptr(), st.cuda_stream)
    torch.cuda.synchronize()
    assert int(flag.item()) == 0
    assert torch.equal(D1, D2)
    ref = A.double() @ B.double().T
    assert rel(D2.cpu().numpy(), ref.cpu().numpy()) < 1e-6


def _data(B, seed=0):
    r = np.random.default_rng(seed)
    X = r.standard_normal((B, DIMS[0])).astype(np.float32)
    Y = r.standard_normal((B, DIMS[-1])).astype(np.float32)
    return X, Y


def test_forward_and_gradients_match_oracle():
    import torch

    net = T.WarmStartMLP(DIMS, max_batch=512, seed=3)
    p = net.GetParams()
    X, Y = _data(384)
    dx, dy = torch.tensor(X, device="cuda"), torch.tensor(Y, device="cuda")
    out = torch.zeros(384, DIMS[-1], device="cuda")
    torch.cuda.synchronize()  # the network runs on its own stream
    net.Forward(dx.data_ptr(), 384, out.data_ptr())
    orc = MO.MLP(DIMS, p, bf16=True)
    y_ref = orc.forward(X)[0]
    assert rel(out.cpu().numpy(), y_ref) < 2e-3
    loss = net.LossGrad(dx.data_ptr(), dy.data_ptr(), 384)
    g = net.GetGrads()
    loss_ref, g_ref = orc.loss_grad(X, Y)
    assert abs(loss - loss_ref) / loss_ref < 1e-3
    assert rel(g, g_ref) < 1e-2
    # layer by layer, the largest gradients agree closely
    Wg, bg = MO.unflatten(g, DIMS)
    Wr, br = MO.unflatten(g_ref, DIMS)
    for l in range(len(DIMS) - 1):
        assert rel(Wg[l], Wr[l]) < 2e-2 and rel(bg[l], br[l]) < 2e-2
    net.Destroy()


def test_adamw_step_matches_oracle():
    import torch

    net = T.WarmStartMLP(DIMS, max_batch=256, seed=5)
    p0 = net.GetParams().astype(np.float64)
    X, Y = _data(256, 1)
    dx, dy = torch.tensor(X, device="cuda"), torch.tensor(Y, device="cuda")
    net.LossGrad(dx.data_ptr(), dy.data_ptr(), 256)
    g = net.GetGrads().astype(np.float64)
    net.AdamWStep(1e-3, 0.9, 0.999, 1e-8, 1e-4)
    p1 = net.GetParams().astype(np.float64)
    z = np.zeros_like(p0)
    p1_ref, _, _ = MO.adamw(p0, g, z, z, 1, 1e-3, 0.9, 0.999, 1e-8, 1e-4, DIMS)
    assert np.max(np.abs(p1 - p1_ref)) < 1e-6
    net.Destroy()


def test_training_fits_a_smooth_map_and_is_deterministic():
    import torch

    r = np.random.default_rng(7)
    X = r.uniform(-1, 1, (1024, DIMS[0])).astype(np.float32)
    Wt = r.standard_normal((DIMS[0], DIMS[-1])) / np.sqrt(DIMS[0])
    Y = np.sin(X @ Wt).astype(np.float32)
    dx, dy = torch.tensor(X, device="cuda"), torch.tensor(Y, device="cuda")

    def run():
        net = T.WarmStartMLP(DIMS, max_batch=256, seed=11)
        first = None
        for ep in range(60):
            for b in range(4):
                xs = dx[256 * b:256 * (b + 1)]
                ys = dy[256 * b:256 * (b + 1)]
                l = net.TrainStep(xs.data_ptr(), ys.data_ptr(), 256, lr=2e-3, want_loss=(ep == 0 and b == 0))
                if first is None:
                    first = l
        last = net.LossGrad(dx[:256].data_ptr(), dy[:256].data_ptr(), 256)
        p = net.GetParams()
        net.Destroy()
        return first, last, p

    first, last, p1 = run()
    assert last < 0.05 * first
    _, last2, p2 = run()
    assert np.array_equal(p1, p2) and last == last2
