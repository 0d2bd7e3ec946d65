"""CPU oracle of the learned patch proposal -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline may use this module, as a
checker; nothing in the product imports it.  It restates, in torch float64 on the CPU, the
proposal move that the CUDA kernels of ising_b200/csrc/learned.cu implement.  The reference
(SamuelJosephs/ISING) has no learned move: its Metropolis_mcs (src/energyMin.f90:234-374)
only proposes single-spin moves.  The parts that are the reference's are the Hamiltonian
terms of the patch energy: calculateHeisenbergEnergy (src/energyMin.f90:86-171), with bulk
DMI D_ij = Dz * r_hat, r_hat = (r_i - r_j)/|r_i - r_j| (:138).

Window: 8^3 sites (a 4^3 patch plus a 2-site halo), 3 channels (Sx, Sy, Sz), indexed
[c][i][j][k] with window site (i, j, k) = lattice site (px - 2 + i, py - 2 + j, pz - 2 + k)
(periodic) for a patch whose lowest corner is (px, py, pz).  Network: conv 3->32 (3^3,
valid, 8^3 -> 6^3), conv 32->32 (valid, 6^3 -> 4^3), conv 32->32 (3^3, zero padding 1,
4^3 -> 4^3), each followed by GELU (tanh form), then a 1^3 head 32 -> 4: a 3-vector mu and
log sigma for each of the 64 patch sites (site order i, j, k with k fastest).

Move: in the tangent frame (e1, e2) of each patch spin s (frame() below) the proposal is
omega = P_s(mu) + sigma * eps, eps ~ N(0, I_2), s' = cos|omega| s + sin|omega| omega/|omega|
(exponential map), and a move with any |omega| >= pi is rejected.  The density of s' has the
Jacobian |omega|/sin|omega|.  The reverse move uses omega_rev = log_{s'}(s) with the network
evaluated on the proposed window.  The acceptance is
min(1, exp(-beta dE_patch) q(x | x') / q(x' | x)).
"""
from __future__ import annotations

import math

import torch

F64 = torch.float64
N_PARAMS = 32 * 3 * 27 + 32 + 32 * 32 * 27 + 32 + 32 * 32 * 27 + 32 + 4 * 32 + 4
PARAM_SHAPES = [("W1", (32, 3, 3, 3, 3)), ("b1", (32,)), ("W2", (32, 32, 3, 3, 3)), ("b2", (32,)),
                ("W3", (32, 32, 3, 3, 3)), ("b3", (32,)), ("Wh", (4, 32)), ("bh", (4,))]


def unflatten(flat) -> dict:
    flat = torch.as_tensor(flat, dtype=F64)
    out, o = {}, 0
    for name, shp in PARAM_SHAPES:
        n = math.prod(shp)
        out[name] = flat[o:o + n].reshape(shp).clone()
        o += n
    assert o == flat.numel()
    return out


def flatten(p: dict) -> torch.Tensor:
    return torch.cat([p[name].reshape(-1) for name, _ in PARAM_SHAPES])


def bf16(t):
    return t.to(torch.bfloat16).to(F64)


def gelu(x):
    return torch.nn.functional.gelu(x, approximate="tanh")


def forward(p: dict, windows, round_bf16: bool = False):
    """windows [B, 3, 8, 8, 8] -> out [B, 64, 4] (mu_x, mu_y, mu_z, log sigma).
    round_bf16 mirrors the device: BF16 weights, inputs and stored activations."""
    r = bf16 if round_bf16 else (lambda t: t)
    x = r(torch.as_tensor(windows, dtype=F64))
    h1 = r(gelu(torch.nn.functional.conv3d(x, r(p["W1"]), p["b1"])))
    h2 = r(gelu(torch.nn.functional.conv3d(h1, r(p["W2"]), p["b2"])))
    h3 = r(gelu(torch.nn.functional.conv3d(h2, r(p["W3"]), p["b3"], padding=1)))
    out = torch.einsum("bcxyz,oc->bxyzo", h3, p["Wh"]) + p["bh"]
    return out.reshape(out.shape[0], 64, 4)


def frame(s):
    """Orthonormal tangent frame (e1, e2) at unit vectors s [..., 3]: helper axis z (x when
    |s_z| >= 0.9), e1 = normalize(a x s), e2 = s x e1."""
    a = torch.zeros_like(s)
    use_x = s[..., 2].abs() >= 0.9
    a[..., 2] = torch.where(use_x, 0.0, 1.0).to(s.dtype)
    a[..., 0] = torch.where(use_x, 1.0, 0.0).to(s.dtype)
    e1 = torch.linalg.cross(a, s, dim=-1)
    e1 = e1 / e1.norm(dim=-1, keepdim=True)
    e2 = torch.linalg.cross(s, e1, dim=-1)
    return e1, e2


def log_map(s, t):
    """omega = log_s(t) as tangent components in the frame of s, and its angle."""
    c = (s * t).sum(-1).clamp(-1.0, 1.0)
    th = torch.arccos(c)
    v = t - c[..., None] * s
    nv = v.norm(dim=-1)
    scale = torch.where(nv > 1e-12, th / nv.clamp_min(1e-300), torch.zeros_like(nv))
    w = v * scale[..., None]
    e1, e2 = frame(s)
    return torch.stack([(w * e1).sum(-1), (w * e2).sum(-1)], -1), th


def exp_map(s, om):
    e1, e2 = frame(s)
    w = om[..., 0:1] * e1 + om[..., 1:2] * e2
    th = w.norm(dim=-1, keepdim=True)
    safe = th.clamp_min(1e-300)
    return torch.where(th > 0, torch.cos(th) * s + torch.sin(th) * w / safe, s)


def tangent_mean(out, s):
    e1, e2 = frame(s)
    mu = out[..., 0:3]
    return torch.stack([(mu * e1).sum(-1), (mu * e2).sum(-1)], -1)


def log_jac(th):
    """log(|omega| / sin|omega|), 0 at omega = 0."""
    return torch.where(th > 1e-6, torch.log(th / torch.sin(th)), th * th / 6.0)


def propose(out, s, eps):
    """out [..., 64, 4] at x, patch spins s [..., 64, 3], noise eps [..., 64, 2] ->
    (s', log q(x'|x) summed over the patch, rejected flag)."""
    m = tangent_mean(out, s)
    ls = out[..., 3]
    sig = torch.exp(ls)
    om = m + sig[..., None] * eps
    th = om.norm(dim=-1)
    rej = (th >= math.pi).any(-1)
    sp = exp_map(s, om)
    lq = (-0.5 * (eps * eps).sum(-1) - 2.0 * ls - math.log(2 * math.pi) + log_jac(th)).sum(-1)
    return sp, lq, rej


def log_q_reverse(out_p, sp, s):
    """log q(x|x') with the network output out_p at x'."""
    om, th = log_map(sp, s)
    m = tangent_mean(out_p, sp)
    ls = out_p[..., 3]
    r = om - m
    return (-0.5 * (r * r).sum(-1) * torch.exp(-2.0 * ls) - 2.0 * ls - math.log(2 * math.pi) + log_jac(th)).sum(-1)


def patch_energy(win, J, D, B, K=0.0, kaxis=(0.0, 0.0, 1.0)):
    """Energy of the 4^3 patch of windows win [..., 3, 8, 8, 8] in the reference's local form:
    sum over patch sites i of sum_j w_ij (J S_i.S_j + D_ij.(S_i x S_j)) - B S_iz - K (S_i.e)^2,
    w_ij = 1/2 for j in the patch, 1 for halo sites; bulk D_ij = -D e_d for j = i + e_d."""
    S = torch.as_tensor(win, dtype=F64)
    P = S[..., 2:6, 2:6, 2:6]
    e = torch.zeros(S.shape[:-4], dtype=F64)
    ka = torch.tensor(kaxis, dtype=F64)
    for d in range(3):
        for sgn in (1, -1):
            sl = [slice(2, 6)] * 3
            sl[d] = slice(2 + sgn, 6 + sgn)
            Nb = S[(...,) + (slice(None),) + tuple(sl)]
            w = torch.ones((4, 4, 4), dtype=F64)
            idx = [slice(None)] * 3
            # neighbours inside the patch carry weight 1/2
            if sgn == 1:
                idx[d] = slice(0, 3)
            else:
                idx[d] = slice(1, 4)
            w[tuple(idx)] = 0.5
            Dv = torch.zeros(3, dtype=F64)
            Dv[d] = -D * sgn
            cr = torch.linalg.cross(P, Nb, dim=-4)
            bond = J * (P * Nb).sum(-4) + (cr * Dv.view(3, 1, 1, 1)).sum(-4)
            e = e + (w * bond).sum((-1, -2, -3))
    e = e - B * P[..., 2, :, :, :].sum((-1, -2, -3))
    if K != 0.0:
        proj = (P * ka.view(3, 1, 1, 1)).sum(-4)
        e = e - K * (proj * proj).sum((-1, -2, -3))
    return e


def patch_spins(win):
    """[..., 3, 8, 8, 8] -> patch spins [..., 64, 3] in (i, j, k) order."""
    P = torch.as_tensor(win, dtype=F64)[..., 2:6, 2:6, 2:6]
    return P.reshape(*P.shape[:-4], 3, 64).transpose(-1, -2)


def loss(p: dict, windows, targets, round_bf16=False):
    """Mean Gaussian negative log-likelihood (up to a constant) of the target patch spins
    [B, 64, 3] under the proposal from windows: 0.5 |log_s(t) - P_s(mu)|^2 / sigma^2 + 2 log sigma."""
    out = forward(p, windows, round_bf16)
    s = patch_spins(windows)
    om, _ = log_map(s, torch.as_tensor(targets, dtype=F64))
    r = om - tangent_mean(out, s)
    ls = out[..., 3].clamp(-6.0, 1.5)        # the proposal's log sigma range (no gradient outside)
    return (0.5 * (r * r).sum(-1) * torch.exp(-2.0 * ls) + 2.0 * ls).mean()


def grads(p: dict, windows, targets, round_bf16=False):
    q = {k: v.clone().requires_grad_(True) for k, v in p.items()}
    L = loss(q, windows, targets, round_bf16)
    L.backward()
    return float(L.detach()), {k: v.grad.detach() for k, v in q.items()}
