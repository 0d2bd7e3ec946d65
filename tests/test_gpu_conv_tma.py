"""The TMA-fed tensor-core convolutions (conv_tma.cu) against the register-staged one
(gemm_umma.cu) and a float32 torch conv3d: 3^3 kernels over 32-channel grids onto 4^3
outputs, valid (6^3 input) and same (4^3 input) padding, odd window counts (a block with one
window), N = 16 / 32 / 64; and the first layer over 8 channels onto 6^3 outputs.  Both tensor-core paths accumulate offset by offset in the same K
order, so their outputs are bit-identical; against float32 the tolerance is 2e-3 of the
output scale (BF16 inputs, FP32 accumulation in a different order)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _conv(ib, x, w, bias, N, Gi, pad, loader, gelu, Go=4):
    import torch
    nwin, ch = x.shape[0], x.shape[-1]
    rows = nwin * Go ** 3
    out_c = torch.empty((rows, N), dtype=torch.float32, device="cuda")
    out_o = torch.empty((rows, N), dtype=torch.bfloat16, device="cuda")
    ib._lib.call("ising_conv3_bf16", C.c_void_p(x.data_ptr()), ch, Gi, Go, pad, nwin, C.c_void_p(w.data_ptr()),
                 w.shape[1], N, C.c_void_p(bias.data_ptr()), C.c_void_p(out_c.data_ptr()), N,
                 C.c_void_p(out_o.data_ptr()), N, gelu, loader, None)
    torch.cuda.synchronize()
    return out_c, out_o


@pytest.mark.parametrize("Gi,pad", [(6, 0), (4, 1)])
@pytest.mark.parametrize("nwin,N", [(1, 32), (2, 32), (5, 32), (3, 16), (4, 64)])
def test_conv_tma_matches_register_path_and_torch(ib, cuda_ok, Gi, pad, nwin, N):
    import torch
    import torch.nn.functional as F
    g = torch.Generator(device="cpu").manual_seed(nwin * 100 + N + Gi)
    x = torch.randn((nwin, Gi, Gi, Gi, 32), generator=g).bfloat16().cuda()
    w = (0.05 * torch.randn((N, 864), generator=g)).bfloat16().cuda()
    bias = torch.randn(N, generator=g).float().cuda()
    c2, o2 = _conv(ib, x, w, bias, N, Gi, pad, loader=2, gelu=1)
    c1, o1 = _conv(ib, x, w, bias, N, Gi, pad, loader=1, gelu=1)
    assert torch.equal(c1, c2)
    assert torch.equal(o1, o2)
    # float32 reference: weight[n, c, dx, dy, dz] = w[n, (9 dx + 3 dy + dz) 32 + c]
    wt = w.float().reshape(N, 3, 3, 3, 32).permute(0, 4, 1, 2, 3).contiguous()
    ref = F.conv3d(x.float().permute(0, 4, 1, 2, 3), wt, bias=bias, padding=pad)
    ref = ref.permute(0, 2, 3, 4, 1).reshape(nwin * 64, N)
    scale = ref.abs().max().item()
    assert (c2 - ref).abs().max().item() <= 2e-3 * scale


@pytest.mark.parametrize("nwin,N", [(1, 32), (3, 32), (7, 32), (2, 16), (3, 64)])
def test_first_layer_tma_matches_register_path_and_torch(ib, cuda_ok, nwin, N):
    """The first layer: 8 (padded) channels, 8^3 -> 6^3 valid, 216 rows per window in a
    256-row tile; K = 27 x 8 padded to 224 (the pad columns meet zeros on both paths)."""
    import torch
    import torch.nn.functional as F
    g = torch.Generator(device="cpu").manual_seed(nwin * 10 + N)
    x = torch.randn((nwin, 8, 8, 8, 8), generator=g).bfloat16().cuda()
    w = (0.1 * torch.randn((N, 224), generator=g)).bfloat16().cuda()
    bias = torch.randn(N, generator=g).float().cuda()
    c2, o2 = _conv(ib, x, w, bias, N, 8, 0, loader=2, gelu=1, Go=6)
    c1, o1 = _conv(ib, x, w, bias, N, 8, 0, loader=1, gelu=1, Go=6)
    assert torch.equal(c1, c2)
    assert torch.equal(o1, o2)
    wt = w[:, :216].float().reshape(N, 3, 3, 3, 8).permute(0, 4, 1, 2, 3).contiguous()
    ref = F.conv3d(x.float().permute(0, 4, 1, 2, 3), wt, bias=bias)
    ref = ref.permute(0, 2, 3, 4, 1).reshape(nwin * 216, N)
    assert (c2 - ref).abs().max().item() <= 2e-3 * ref.abs().max().item()


def test_conv_tma_rejects_other_shapes(ib, cuda_ok):
    """The input gradient of the second layer (32 channels, 4^3 -> 6^3, pad 2) has no TMA
    form: loader 2 refuses it before any launch, the register-staged path takes it."""
    import torch
    x = torch.zeros((2, 4, 4, 4, 32), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((32, 864), dtype=torch.bfloat16, device="cuda")
    b = torch.zeros(32, dtype=torch.float32, device="cuda")
    out = torch.empty((2 * 216, 32), dtype=torch.float32, device="cuda")
    with pytest.raises(ib.IsingError):
        ib._lib.call("ising_conv3_bf16", C.c_void_p(x.data_ptr()), 32, 4, 6, 2, 2, C.c_void_p(w.data_ptr()), 864, 32,
                     C.c_void_p(b.data_ptr()), C.c_void_p(out.data_ptr()), 32, None, 0, 0, 2, None)
    ib._lib.call("ising_conv3_bf16", C.c_void_p(x.data_ptr()), 32, 4, 6, 2, 2, C.c_void_p(w.data_ptr()), 864, 32,
                 C.c_void_p(b.data_ptr()), C.c_void_p(out.data_ptr()), 32, None, 0, 0, 1, None)
