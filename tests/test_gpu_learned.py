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


def _rand_windows(n, seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    w = torch.randn((n, 3, 8, 8, 8), generator=g, dtype=torch.float64)
    w[:, 2] += 1.5                                   # partly ordered along +z
    return w / w.norm(dim=1, keepdim=True)


def _targets(windows, seed, amp=0.3):
    import torch
    from oracle import learned_ref as R
    g = torch.Generator().manual_seed(seed)
    s = R.patch_spins(windows)
    om = amp * torch.randn(s.shape[:-1] + (2,), generator=g, dtype=torch.float64)
    return R.exp_map(s, om)


def test_network_forward_matches_oracle(ib, cuda_ok):
    import torch
    from oracle import learned_ref as R
    net = ib.ProposalNet(max_batch=8, seed=3)
    p = R.unflatten(net.get_params())
    p["bh"][:3] = torch.tensor([0.1, -0.2, 0.05], dtype=torch.float64)
    net.set_params(R.flatten(p).numpy())
    w = _rand_windows(6, 1)
    out = net.forward(w.float().cuda()).double().cpu()
    # the oracle sees the same FP32-rounded windows and BF16 weights / activations
    ref = R.forward(R.unflatten(net.get_params()), w.float().double(), round_bf16=True)
    err = (out - ref).abs().max().item()
    assert err <= 2e-2 * ref.abs().max().item() + 2e-3, err


def test_network_gradients_match_oracle(ib, cuda_ok):
    import torch
    from oracle import learned_ref as R
    net = ib.ProposalNet(max_batch=8, seed=5)
    w = _rand_windows(8, 2)
    t = _targets(w, 3)
    loss, g = net.loss_grad(w.float().cuda(), t.float().cuda())
    p = R.unflatten(net.get_params())
    lref, gref = R.grads(p, w.float().double(), t.float().double(), round_bf16=True)
    assert abs(loss - lref) <= 1e-2 * abs(lref) + 1e-3, (loss, lref)
    G = R.unflatten(g)
    for name, _ in R.PARAM_SHAPES:
        a, b = G[name].reshape(-1), gref[name].reshape(-1)
        rel = (a - b).norm() / b.norm().clamp_min(1e-12)
        assert rel < 5e-2, (name, float(rel))


def test_training_reduces_the_loss(ib, cuda_ok):
    import torch
    from oracle import learned_ref as R
    net = ib.ProposalNet(max_batch=64, seed=7)
    w = _rand_windows(64, 4)
    s = R.patch_spins(w)
    # a learnable target: rotate every patch spin by 0.4 rad toward +z in its tangent frame
    e1, e2 = R.frame(s)
    ez = torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64)
    om = torch.stack([(ez * e1).sum(-1), (ez * e2).sum(-1)], -1)
    om = 0.4 * om / om.norm(dim=-1, keepdim=True).clamp_min(1e-9)
    t = R.exp_map(s, om)
    wc, tc = w.float().cuda(), t.float().cuda()
    l0 = net.train_step(wc, tc, lr=3e-3)
    for _ in range(150):
        l1 = net.train_step(wc, tc, lr=3e-3)
    assert np.isfinite(l1) and l1 < l0 - 1.0, (l0, l1)
