"""The proposal density of the learned patch move, checked from first principles on the CPU
(the device's densities equal the oracle's, tests/test_gpu_learned.py): for a source spin s
and a network output (mean rotation mu, log sigma), the density q(t|s) that enters the
Metropolis-Hastings ratio, evaluated through log_q_reverse (the tangent Gaussian at s, the
exponential map's Jacobian |omega| / sin|omega|), must

- integrate over the sphere to the probability that a draw is not rejected (|omega| < pi):
  checked by Monte Carlo over uniform targets against the rejection rate of the draws;
- equal, at every proposed target, the forward density the proposal itself records (propose:
  the noise of the draw plus the same Jacobian), which ties the exponential and logarithm maps
  and the frames together.

A wrong Jacobian, a missing factor of the Gaussian's normalisation or mismatched frames break
the first (the integral moves away from the acceptance mass) or the second."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _case(seed, sig, mu_len, n_src):
    g = torch.Generator().manual_seed(seed)
    s = torch.randn(n_src, 1, 3, generator=g, dtype=torch.float64)
    s = s / s.norm(dim=-1, keepdim=True)
    mu = torch.randn(n_src, 1, 3, generator=g, dtype=torch.float64)
    mu = mu / mu.norm(dim=-1, keepdim=True) * mu_len
    out = torch.cat([mu, torch.full((n_src, 1, 1), math.log(sig), dtype=torch.float64)], -1)
    return s, out, g


@pytest.mark.parametrize("sig,mu_len", [(0.3, 0.0), (0.5, 0.4), (0.9, 0.8), (1.4, 0.0)])
def test_density_integrates_to_the_acceptance_mass(sig, mu_len):
    from oracle import learned_ref as R
    s, out, g = _case(11, sig, mu_len, 4)
    n = 400000
    for k in range(s.shape[0]):
        src = s[k:k + 1].expand(n, 1, 3)
        o = out[k:k + 1].expand(n, 1, 4)
        t = torch.randn(n, 1, 3, generator=g, dtype=torch.float64)
        t = t / t.norm(dim=-1, keepdim=True)
        # integral over the sphere = 4 pi E_uniform[q(t|s)]; the oracle's log densities carry
        # -log(2 pi) per site, the Gaussian's normalisation
        q = torch.exp(R.log_q_reverse(o, src, t))
        integral = float(4 * math.pi * q.mean())
        se = float(4 * math.pi * q.std() / math.sqrt(n))
        eps = torch.randn(n, 1, 2, generator=g, dtype=torch.float64)
        _, _, rej = R.propose(o, src, eps)
        kept = 1.0 - float(rej.double().mean())
        assert abs(integral - kept) < 5 * se + 3e-3, (sig, mu_len, k, integral, kept, se)


@pytest.mark.parametrize("sig,mu_len", [(0.3, 0.2), (0.9, 0.8), (1.4, 1.0)])
def test_forward_density_equals_density_at_the_proposed_target(sig, mu_len):
    from oracle import learned_ref as R
    s, out, g = _case(5, sig, mu_len, 2000)
    eps = torch.randn(s.shape[0], 1, 2, generator=g, dtype=torch.float64)
    sp, lq, rej = R.propose(out, s, eps)
    keep = ~rej
    lq_eval = R.log_q_reverse(out, s, sp)       # density of target sp from source s, output at s
    assert torch.allclose(lq[keep], lq_eval[keep], atol=1e-8, rtol=0), \
        float((lq[keep] - lq_eval[keep]).abs().max())
