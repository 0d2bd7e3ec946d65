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


# ---------------------------------------------------------------- the patch move
def _pt_setup(ib, L=8, betas=(0.1, 0.3, 1.0, 3.0), J=-1.0, D=0.5, B=0.25, K=0.0, seed=11, record=0):
    m = ib.ChainMesh.simple_cubic(L, n_replicas=len(betas))
    m.init_uniform(seed, 0)
    p = ib.params(J=J, Dz=D, B=B, K=K, dmi="bulk", include_Jp=False)
    pt = ib.ParallelTempering(m, np.array(betas), p, seed=seed, ensemble=0, record=bool(record), record_capacity=record)
    return m, p, pt


def _window(spins, L, origin):
    """[3, 8, 8, 8] window of a (3, L^3) spin array (reference atom order, z fastest)."""
    S = spins.reshape(3, L, L, L)
    idx = [(np.arange(8) + o - 2) % L for o in origin]
    return S[:, idx[0]][:, :, idx[1]][:, :, :, idx[2]]


def test_patch_move_matches_oracle(ib, cuda_ok):
    import torch
    from oracle import learned_ref as R
    L, betas = 8, (0.1, 0.3, 1.0, 3.0)
    m, p, pt = _pt_setup(ib, L, betas)
    net = ib.ProposalNet(max_batch=16, seed=9)
    params = R.unflatten(net.get_params())
    colour, off = 5, (1, 2, 3)
    scale = np.array([0.5, 1.0, 0.25, 0.1], np.float32)
    drift = 0.7
    pt.patch_set_scale(scale, drift)
    t2r = pt.permutation()
    pre = [m.get_spins(r).T.copy() for r in range(len(betas))]          # (3, N)
    pt.patch_step(net, colour, off)
    post = [m.get_spins(r).T.copy() for r in range(len(betas))]
    n = len(betas)
    win = np.empty((n, 3, 8, 8, 8), np.float32)
    winp = np.empty((n, 3, 8, 8, 8), np.float32)
    lqf = np.empty(n)
    dE = np.empty(n)
    acc = np.empty(n, np.int32)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ib._lib.call("ising_pt_patch_last", pt._h, n, fp(win), fp(winp), dp(lqf), dp(dE), acc.ctypes.data_as(C.POINTER(C.c_int)))
    origin = ((4 * (colour & 1) + off[0]) % L, (4 * ((colour >> 1) & 1) + off[1]) % L, (4 * ((colour >> 2) & 1) + off[2]) % L)
    n_acc = 0
    for t in range(n):
        r = t2r[t]
        x = torch.tensor(win[t], dtype=torch.float64)
        xp = torch.tensor(winp[t], dtype=torch.float64)
        np.testing.assert_array_equal(win[t], _window(pre[r], L, origin).astype(np.float32))
        halo = np.ones((8, 8, 8), bool)
        halo[2:6, 2:6, 2:6] = False
        np.testing.assert_array_equal(winp[t][:, halo], win[t][:, halo])
        s, sp = R.patch_spins(x), R.patch_spins(xp)
        assert torch.allclose(sp.norm(dim=-1), torch.ones(64, dtype=torch.float64), atol=1e-5)
        out = R.forward(params, x[None], round_bf16=True)[0]
        outp = R.forward(params, xp[None], round_bf16=True)[0]
        om, th = R.log_map(s, sp)
        a = float(scale[t])
        ls = out[:, 3].clamp(-6.0, 1.5) + np.log(a)
        eps = (om - a * drift * R.tangent_mean(out, s)) / torch.exp(ls)[:, None]
        lq_f = float((-0.5 * (eps * eps).sum(-1) - 2.0 * ls + R.log_jac(th)).sum())
        outp_c = outp.clone()
        outp_c[:, :3] *= a * drift
        outp_c[:, 3] = outp_c[:, 3].clamp(-6.0, 1.5) + np.log(a)
        lq_r = float(R.log_q_reverse(outp_c, sp, s)) + 64 * np.log(2 * np.pi)
        de = float(R.patch_energy(xp, -1.0, 0.5, 0.25) - R.patch_energy(x, -1.0, 0.5, 0.25))
        assert abs(lq_f - lqf[t]) < 0.5, (lq_f, lqf[t])
        assert abs(de - dE[t]) < 1e-3 * max(1.0, abs(de)) or not acc[t], (de, dE[t])
        la = -betas[t] * de + lq_r - lq_f
        if la > 3.0 and float(th.max()) < np.pi - 1e-3:
            assert acc[t] == 1, (t, la)
        if la < -30.0:
            assert acc[t] == 0, (t, la)
        # spins after the step: the patch is x' when accepted, x otherwise; nothing else moved
        expect = pre[r].copy().reshape(3, L, L, L)
        if acc[t]:
            n_acc += 1
            idx = [(np.arange(2, 6) + o - 2) % L for o in origin]
            expect[np.ix_(range(3), idx[0], idx[1], idx[2])] = winp[t][:, 2:6, 2:6, 2:6]
        np.testing.assert_allclose(post[r].reshape(3, L, L, L), expect, atol=0, rtol=0)
    proposed, accepted = pt.patch_stats()
    assert proposed.sum() == n and accepted.sum() == n_acc


def test_patch_steps_keep_the_running_energies(ib, cuda_ok):
    m, p, pt = _pt_setup(ib, 16, (0.2, 0.5, 1.0), K=0.05)
    net = ib.ProposalNet(max_batch=64, seed=2)
    rng = np.random.default_rng(0)
    for i in range(12):
        pt.run(1, 1)
        pt.patch_step(net, i % 8, tuple(int(v) for v in rng.integers(0, 4, 3)))
    e_run, m_run = pt.energies()
    pt.resync()
    e_new, m_new = pt.energies()
    assert np.max(np.abs(e_run - e_new)) < 1e-6 * 16 ** 3
    assert np.max(np.abs(m_run - m_new)) < 1e-6 * 16 ** 3
    assert pt.patch_stats()[0].sum() == 12 * 3 * 8


def test_patch_samples(ib, cuda_ok):
    import torch
    m, p, pt = _pt_setup(ib, 8, (0.5, 2.0))
    w, t = pt.patch_samples(2, (0, 1, 2), n_local=0)
    assert w.shape == (2, 3, 8, 8, 8) and t.shape == (2, 64, 3)
    from oracle import learned_ref as R
    np.testing.assert_array_equal(R.patch_spins(w.double().cpu()).numpy(), t.double().cpu().numpy())
    w2, t2 = pt.patch_samples(2, (0, 1, 2), n_local=30)
    np.testing.assert_array_equal(w2.cpu().numpy(), w.cpu().numpy())        # the state is not changed
    assert torch.allclose(t2.norm(dim=-1), torch.ones_like(t2[..., 0]), atol=1e-5)
    assert (t2 - t).abs().max().item() > 0.1


def test_patch_moves_leave_the_energy_distribution_unchanged(ib, cuda_ok):
    """Plain Metropolis vs Metropolis alternating with patch moves on a small lattice: the
    mean energy agrees within four binning standard errors."""
    from ising_b200.analysis import binning_error
    means = []
    for learned in (False, True):
        m, p, pt = _pt_setup(ib, 8, (0.8,), D=0.3, B=0.1, seed=21 + learned, record=3000)
        net = ib.ProposalNet(max_batch=16, seed=4)
        rng = np.random.default_rng(1)
        for i in range(3000):
            pt.run(1, 1)
            if learned:
                pt.patch_step(net, int(rng.integers(0, 8)), tuple(int(v) for v in rng.integers(0, 8, 3)))
        e = pt.series()[0, 500:, 0]
        means.append((e.mean(), binning_error(e)))
        if learned:
            assert pt.patch_stats()[1].sum() > 0
    (a, ea), (b, eb) = means
    assert abs(a - b) < 4.0 * np.hypot(ea, eb), means


def test_trained_network_gains_over_the_untrained_proposal(ib, cuda_ok):
    """What training buys: at the same tuned acceptance (~25%), the trained proposal moves
    the patch spins further per proposal (expected squared jump distance, ESJD) than the
    network as initialised (zero mean rotation, sigma = 0.3 everywhere): here at least 1.5x
    after 300 Adam steps on a 16^3 lattice (16x on the 96^3 C5 ensemble with 1e5 windows)."""
    import torch
    torch.manual_seed(0)
    m, p, pt = _pt_setup(ib, 16, (0.5, 1.0, 2.0, 4.0), D=0.5, B=0.25, seed=3)
    pt.relax(300)

    def esjd(net, drift):
        pt.patch_tune_scale(net, target=0.25, iters=8, seed=5, drift=drift)
        p0, a0 = pt.patch_stats()
        j0 = pt.patch_jump()
        for c in range(8):
            pt.patch_step(net, c, (c % 4, (c + 1) % 4, (c + 2) % 4))
        p1, a1 = pt.patch_stats()
        j1 = pt.patch_jump()
        return float(((j1 - j0) / np.maximum(p1 - p0, 1)).mean()), float(((a1 - a0) / np.maximum(p1 - p0, 1)).mean())

    net0 = ib.ProposalNet(max_batch=64, seed=11)
    e0, acc0 = esjd(net0, 1.0)
    net = ib.ProposalNet(max_batch=256, seed=11)
    ws, ts = [], []
    rng = np.random.default_rng(0)
    for i in range(40):
        pt.relax(5)
        w, t = pt.patch_samples(int(rng.integers(0, 8)), tuple(int(v) for v in rng.integers(0, 8, 3)), n_local=100)
        ws.append(w)
        ts.append(t)
    W, T = torch.cat(ws), torch.cat(ts)
    for step in range(300):
        j = torch.randint(0, W.shape[0], (256,), device=W.device)
        net.train_step(W[j], T[j], lr=1e-3)
    e1, acc1 = esjd(net, 0.25)
    assert 0.1 < acc0 < 0.5 and 0.1 < acc1 < 0.5, (acc0, acc1)
    assert e1 > 1.5 * e0, (e0, e1)


def test_learned_only_chains_sample_the_boltzmann_distribution(ib, cuda_ok):
    """Stationarity of the learned move by itself.  16 replicas of SC L=8 with the C5
    Hamiltonian (bulk D=0.5, B=0.25) at T=1 are equilibrated by 2000 plain sweeps on two twin
    meshes (bit-identical states).  Then one mesh continues with plain single-spin sweeps only
    and the other moves ONLY by learned patch proposals (all eight colour classes per step,
    random offsets), with a network trained so that its mean rotations are non-zero and its
    spreads site-dependent, at drift 0.1 (the trained mean rotation is many sigma long, so a
    larger drift is almost never accepted): the proposal is asymmetric, so the forward and
    reverse densities, the exponential map's Jacobian and the |omega| < pi rejection all enter
    the acceptance.  If the MH ratio is exact, the learned chains stay in the Boltzmann
    distribution the plain chains sample: the per-replica averages of E/N, |M|/N, Q, and the
    per-replica C_v and chi agree (paired over replicas, which share their starting state)
    within 3 standard errors."""
    import torch
    torch.manual_seed(0)
    R, L, beta = 16, 8, 1.0
    N = L ** 3
    p = ib.params(J=-1.0, Dz=0.5, B=0.25, dmi="bulk", include_Jp=False)
    meshes, pts = [], []
    for _ in range(2):
        m = ib.ChainMesh.simple_cubic(L, n_replicas=R)
        m.init_uniform(0xB41, 0)
        meshes.append(m)
        pts.append(ib.ParallelTempering(m, np.full(R, beta), p, seed=0xB41, ensemble=0))
    for pt in pts:
        pt.relax(2000)
    for r in range(R):
        np.testing.assert_array_equal(meshes[0].get_spins(r), meshes[1].get_spins(r))
    plain, learned = pts
    # a trained network: windows of the equilibrated states, targets from local equilibration
    net = ib.ProposalNet(max_batch=64, seed=13)
    rng = np.random.default_rng(3)
    ws, ts = [], []
    for i in range(24):
        w, t = learned.patch_samples(int(rng.integers(0, 8)), tuple(int(v) for v in rng.integers(0, 8, 3)), n_local=20)
        ws.append(w)
        ts.append(t)
    W, T = torch.cat(ws), torch.cat(ts)
    for step in range(200):
        j = torch.randint(0, W.shape[0], (64,), device=W.device)
        net.train_step(W[j], T[j], lr=2e-3)
    out = net.forward(W[:64]).float()
    assert out[..., :3].abs().mean().item() > 1e-2          # non-zero mean rotations
    learned.patch_tune_scale(net, target=0.3, iters=10, seed=4, drift=0.1)
    # the tuning steps moved the learned arm only; both arms now run n_meas steps
    n_meas = 2500
    q = C.c_double()

    def sample(pt, mesh, with_q):
        e, mv = pt.energies()
        qs = []
        if with_q:
            for r in range(R):
                ib._lib.call("ising_winding_number", mesh.handle, r, L // 2, C.byref(q))
                qs.append(q.value)
        return e / N, np.linalg.norm(mv, axis=1) / N, qs

    series = {0: ([], [], []), 1: ([], [], [])}
    p0, a0 = learned.patch_stats()
    for it in range(n_meas):
        plain.relax(1)
        for c in range(8):
            learned.patch_step(net, c, tuple(int(v) for v in rng.integers(0, 8, 3)))
        for arm, (pt, mesh) in enumerate(((plain, meshes[0]), (learned, meshes[1]))):
            e, mm, qs = sample(pt, mesh, it % 5 == 4)
            series[arm][0].append(e)
            series[arm][1].append(mm)
            if qs:
                series[arm][2].append(qs)
    p1, a1 = learned.patch_stats()
    acc = float((a1 - a0).sum() / max(int((p1 - p0).sum()), 1))
    assert 0.05 < acc < 0.8, acc
    stats = {}
    for arm in (0, 1):
        E, M, Q = (np.array(x).T for x in series[arm])             # [replica][sample]
        stats[arm] = {"E": E.mean(1), "M": M.mean(1), "Q": Q.mean(1),
                      "C_v": beta * beta * N * E.var(1), "chi": beta * N * M.var(1)}
    z = {}
    for k in ("E", "M", "Q", "C_v", "chi"):
        d = stats[1][k] - stats[0][k]
        se = d.std(ddof=1) / np.sqrt(R)
        z[k] = abs(d.mean()) / se if se > 0 else 0.0
    print("learned-only vs plain-only:", {k: round(v, 2) for k, v in z.items()}, "acceptance", round(acc, 3))
    assert max(z.values()) < 3.0, z
