"""Learned patch proposal: the tcgen05 BF16 GEMM, the proposal network's forward and
backward passes against the CPU oracle (oracle/learned_ref.py, torch float64), and the
Metropolis-Hastings patch move."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(ib, A, B, bias=None, gelu=False, want_bf16=False):
    import torch
    M, K = A.shape
    N = B.shape[0]
    Mp = (M + 127) // 128 * 128
    Ap = torch.zeros((Mp, K), dtype=torch.bfloat16, device="cuda")
    Ap[:M] = A
    Cout = torch.empty((M, N), dtype=torch.float32, device="cuda")
    O = torch.empty((M, N), dtype=torch.bfloat16, device="cuda") if want_bf16 else None
    fp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_float)) if t is not None else None
    ib._lib.call("ising_bf16_gemm", C.c_void_p(Ap.data_ptr()), K, C.c_void_p(B.data_ptr()), K, M, N, K, fp(bias),
                 fp(Cout), N, C.c_void_p(O.data_ptr()) if O is not None else None, N, int(gelu),
                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return Cout, O


@pytest.mark.parametrize("M,N,K", [(128, 32, 16), (200, 32, 96), (384, 16, 864), (256, 144, 64), (130, 256, 1024)])
def test_tcgen05_gemm_matches_fp32_matmul(ib, cuda_ok, M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    bias = torch.randn((N,), generator=g, device="cuda")
    Cg, O = _gemm(ib, A, B, bias=bias, gelu=True, want_bf16=True)
    ref = A.double() @ B.double().T + bias.double()
    err = (Cg.double() - ref).abs().max().item()
    assert err <= 1e-4 * np.sqrt(K) * ref.abs().max().item() + 1e-4, err
    gel = torch.nn.functional.gelu(ref, approximate="tanh")
    assert (O.double() - gel).abs().max().item() <= 1e-2 * gel.abs().max().item() + 1e-2
