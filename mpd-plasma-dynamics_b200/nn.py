"""Host side of the surrogate network's device kernels: thin wrappers that
pass torch-allocated device buffers (torch only provides memory and the
stream) to the library's own kernels through the C ABI."""
from __future__ import annotations

import ctypes as C

from . import _native as N


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def gemm(A, B, Cout, M, N_, K, batch=1, sa=None, sb=None, sc=None, alpha=1.0, beta=0.0,
         work=None):
    """Cout[b](m,n) = alpha * sum_k A[b](m,k) B[b](n,k) + beta * Cout[b](m,n) on the
    tcgen05 tensor cores (operands rounded to BF16, FP32 accumulate).
    sa = (row, k, batch) element strides of A (default: row-major M x K
    contiguous), likewise sb for B (N x K) and sc for Cout (M x N).  work: an
    optional float32 device buffer for split-K partial sums."""
    lib = N.load()
    sa = sa or (K, 1, M * K)
    sb = sb or (K, 1, N_ * K)
    sc = sc or (N_, 1, M * N_)
    d = N.GemmDesc(M, N_, K, batch, A.data_ptr(), sa[0], sa[1], sa[2], B.data_ptr(), sb[0],
                   sb[1], sb[2], Cout.data_ptr(), sc[0], sc[1], sc[2], float(alpha), float(beta),
                   work.data_ptr() if work is not None else None,
                   work.numel() if work is not None else 0)
    N.check(lib.mpd_nn_gemm(C.byref(d), _stream()), lib)
    return Cout


def wait_status():
    lib = N.load()
    N.check(lib.mpd_nn_wait_status(_stream()), lib)
