"""The Poisson-likelihood gradient on the B200 (FP32 forward, adjoint kernel) against the float64 oracle's adjoint
and float64 central differences (h = 1e-4 max(1, |theta|)): <= 1e-4 relative; the NLL and expected counts within
1e-5."""
import numpy as np
import pytest
import torch

from insiliscope_b200 import IscuError
from insiliscope_b200.nll import NllModel, NllSpec, poisson_nll
from insiliscope_b200.workloads import nll_counts, nll_rois
from oracle.nll_oracle import NllSpec as OSpec, expected, gradient, nll, tables

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(engine):
    spec = NllSpec()
    model = NllModel(engine, spec)
    prob = nll_rois(seed=7, frames=4, per_frame=24, spec=spec)
    counts = nll_counts(engine, model, prob)
    return model, prob, counts, OSpec(), tables(OSpec())


def _dev(prob, counts):
    return (torch.from_numpy(prob.params).cuda(), torch.from_numpy(prob.frame).cuda(),
            torch.from_numpy(prob.bg).cuda(), counts)


def test_counts_are_poisson_of_expected(problem):
    model, prob, counts, ospec, t = problem
    mu = expected(ospec, prob.params_true.astype(np.float64), prob.frame, prob.bg_true.astype(np.float64),
                  prob.zern_true, t)
    k = counts.cpu().numpy().astype(np.float64)
    assert np.all(k == np.round(k)) and k.min() >= 0
    # the counts scatter about the expectation as Poisson draws do
    z = (k - mu) / np.sqrt(mu)
    assert abs(z.mean()) < 0.05 and 0.9 < z.std() < 1.1


def test_forward_matches_oracle(problem):
    model, prob, counts, ospec, t = problem
    p, fr, bg, k = _dev(prob, counts)
    value, mu, _ = model.evaluate(p, fr, bg, prob.zern, k, want_mu=True)
    pd = prob.params.astype(np.float64)
    want_mu = expected(ospec, pd, prob.frame, prob.bg.astype(np.float64), prob.zern, t)
    got = mu.cpu().numpy()
    assert np.max(np.abs(got - want_mu)) <= 1e-5 * np.max(want_mu)
    want = nll(ospec, pd, prob.frame, prob.bg.astype(np.float64), prob.zern, k.cpu().numpy(), t)
    assert abs(value - want) <= 1e-5 * abs(want)


def test_gradient_matches_oracle_adjoint_and_central_differences(problem):
    model, prob, counts, ospec, t = problem
    p, fr, bg, k = _dev(prob, counts)
    _, _, (gp, gb, gz) = model.evaluate(p, fr, bg, prob.zern, k, grad=True)
    gp, gb, gz = gp.cpu().numpy().astype(np.float64), gb.cpu().numpy(), gz.cpu().numpy()
    pd, bd, kd = prob.params.astype(np.float64), prob.bg.astype(np.float64), k.cpu().numpy().astype(np.float64)
    _, wp, wb, wz = gradient(ospec, pd, prob.frame, bd, prob.zern, kd, t)
    for col in range(4):
        scale = np.max(np.abs(wp[:, col]))
        assert np.max(np.abs(gp[:, col] - wp[:, col])) <= 1e-4 * scale, col
    assert np.max(np.abs(gb - wb)) <= 1e-4 * np.max(np.abs(wb))
    assert np.max(np.abs(gz - wz)) <= 1e-4 * np.max(np.abs(wz))
    # central differences of the float64 NLL on a seeded subset
    rng = np.random.default_rng(3)

    def fd(f, x, i):
        h = 1e-4 * max(1.0, abs(x.flat[i]))
        xp, xm = x.copy(), x.copy()
        xp.flat[i] += h
        xm.flat[i] -= h
        return (f(xp) - f(xm)) / (2 * h)

    for i in rng.choice(pd.size, 12, replace=False):
        d = fd(lambda P: nll(ospec, P, prob.frame, bd, prob.zern, kd, t), pd, i)
        assert abs(gp.flat[i] - d) <= 1e-4 * max(abs(d), 1e-3 * np.max(np.abs(wp[:, i % 4]))), i
    for j in rng.choice(len(prob.zern), 4, replace=False):
        d = fd(lambda Z: nll(ospec, pd, prob.frame, bd, Z, kd, t), prob.zern.copy(), j)
        assert abs(gz[j] - d) <= 1e-4 * max(abs(d), 1e-3 * np.max(np.abs(wz))), j
    d = fd(lambda B: nll(ospec, pd, prob.frame, B, prob.zern, kd, t), bd, 1)
    assert abs(gb[1] - d) <= 1e-4 * abs(d)


def test_autograd_function(problem):
    model, prob, counts, ospec, t = problem
    p, fr, bg, k = _dev(prob, counts)
    p = p.clone().requires_grad_(True)
    bg = bg.clone().requires_grad_(True)
    z = torch.tensor(prob.zern, dtype=torch.float64, requires_grad=True)
    loss = poisson_nll(model, p, bg, z, k, fr)
    (2.0 * loss).backward()
    _, _, (gp, gb, gz) = model.evaluate(p, fr, bg, prob.zern, k, grad=True)
    assert torch.allclose(p.grad, 2.0 * gp, rtol=1e-6, atol=0)
    assert torch.allclose(bg.grad.double(), 2.0 * gb, rtol=1e-6)
    assert torch.allclose(z.grad, 2.0 * gz.cpu(), rtol=1e-12)


def test_bad_frame_reported(problem):
    model, prob, counts, _, _ = problem
    p, fr, bg, k = _dev(prob, counts)
    fr = fr.clone()
    fr[5] = 99
    with pytest.raises(IscuError):
        model.evaluate(p, fr, bg, prob.zern, k)
