"""The surrogate's tcgen05 BF16 GEMM against numpy: operands rounded to BF16
(round to nearest even), products summed in float64, so the only difference
left is the kernel's FP32 accumulation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def ref_gemm(A, B, Cin, alpha, beta):
    out = alpha * np.einsum("bmk,bnk->bmn", bf16(A), bf16(B))
    return out + beta * Cin if beta != 0.0 else out


def check(pkg, M, N, K, batch, trans_a=False, trans_b=False, alpha=1.0, beta=0.0, seed=0,
          work=0):
    import torch
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((batch, M, K)).astype(np.float32)
    B = rng.standard_normal((batch, N, K)).astype(np.float32)
    C0 = rng.standard_normal((batch, M, N)).astype(np.float32)
    # stored transposed where asked: A as (batch, K, M), B as (batch, K, N)
    a_store = np.ascontiguousarray(A.transpose(0, 2, 1)) if trans_a else A
    b_store = np.ascontiguousarray(B.transpose(0, 2, 1)) if trans_b else B
    dA = torch.from_numpy(a_store).cuda()
    dB = torch.from_numpy(b_store).cuda()
    dC = torch.from_numpy(C0.copy()).cuda()
    sa = (1, M, M * K) if trans_a else (K, 1, M * K)
    sb = (1, N, N * K) if trans_b else (K, 1, N * K)
    w = torch.zeros(work, dtype=torch.float32, device="cuda") if work else None
    pkg.nn.gemm(dA, dB, dC, M, N, K, batch, sa=sa, sb=sb, alpha=alpha, beta=beta, work=w)
    pkg.nn.wait_status()
    got = dC.cpu().numpy().astype(np.float64)
    want = ref_gemm(A, B, C0, alpha, beta)
    scale = alpha * np.einsum("bmk,bnk->bmn", np.abs(bf16(A)), np.abs(bf16(B))) + abs(beta) * np.abs(C0) + 1e-30
    err = np.abs(got - want) / scale
    assert err.max() < 2e-6 * max(1.0, np.sqrt(K)), (M, N, K, err.max())


def test_single_tile(pkg):
    check(pkg, 128, 64, 64, 1)


@pytest.mark.parametrize("M,N,K,batch", [(1, 1, 1, 1), (200, 100, 150, 3), (130, 70, 17, 2),
                                         (512, 64, 1024, 1), (64, 200, 256, 5)])
def test_ragged_shapes(pkg, M, N, K, batch):
    check(pkg, M, N, K, batch, seed=M + N + K)


@pytest.mark.parametrize("ta,tb", [(True, False), (False, True), (True, True)])
def test_transposed_operands(pkg, ta, tb):
    check(pkg, 150, 90, 130, 2, trans_a=ta, trans_b=tb, seed=7)


def test_alpha_beta(pkg):
    check(pkg, 140, 80, 96, 2, alpha=0.5, beta=-1.25, seed=3)


@pytest.mark.parametrize("M,N,K,batch,ta", [(256, 64, 4100, 2, False), (64, 64, 4100, 3, True),
                                            (200, 70, 1000, 1, False)])
def test_split_k(pkg, M, N, K, batch, ta):
    """Few output tiles and long K: the sum is split over K (partials summed
    in a fixed order) and must agree with numpy like the unsplit product."""
    check(pkg, M, N, K, batch, trans_a=ta, alpha=0.75, beta=0.5, seed=11, work=64 * M * N * batch)
