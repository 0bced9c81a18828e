"""The checkpointed torch.autograd.Function over the FP64 step.

* dot-product test of 20 steps (remap every 5, checkpoints every 5)
  against the oracle's tangent-linear model, to 1e-12;
* gradient of J = sum(mask * theta^2) at the final step against central
  finite differences of the GPU forward (eps = 1e-6 along random unit
  directions) on a state without limiter ties.
"""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from atmdyn import ic, Dycore
from atmdyn.adjoint import integrate, gaussian_mask
import pyoracle

pytestmark = pytest.mark.gpu

NAMES = ('dp', 'pt', 'ud', 'vd')
STATE = {'dp': pyoracle.DP, 'pt': pyoracle.PT, 'ud': pyoracle.UD, 'vd': pyoracle.VD}
SCALE = {'dp': 10.0, 'pt': 0.01, 'ud': 0.5, 'vd': 0.5}
P0K = 1.0e5 ** ic.KAPPA  # theta = pt * p0**kappa


def small_jet(seed=2, noisy=False):
    st = ic.jet_case(48, 40, 12, 25e3, 25e3, width=200e3, seed=seed)
    st.dt = 30.0
    if noisy:  # no exact ties anywhere (uniform dp, x-independent winds)
        rng = np.random.default_rng(seed + 100)
        st.dp = st.dp + rng.normal(0, 5.0, st.dp.shape)
        st.u = st.u + rng.normal(0, 0.5, st.u.shape)
        st.v = st.v + rng.normal(0, 0.5, st.v.shape)
    return st


def tensors(st):
    return [torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device='cuda', requires_grad=True)
            for a in (st.dp, st.pt, st.u, st.v)]


def test_twenty_steps_dot_product():
    st = small_jet()
    nsteps, remap_every, ckpt = 20, 5, 5
    rng = np.random.default_rng(11)
    v = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    w = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    t = pyoracle.TLMModel(st, v, threads=8)
    for s in range(nsteps):
        t.cgrid_step(st.dt / 2)
        t.cgrid_halo()
        t.dgrid_step(st.dt)
        if (s + 1) % remap_every == 0:
            t.remap()
        t.dgrid_halo()
    lhs = sum(np.sum(w[n] * t.get(STATE[n])[1]) for n in NAMES)
    dyn = Dycore(st)
    dyn.adj_enable()
    x = tensors(st)
    y = integrate(dyn, x, nsteps, st.dt, remap_every, ckpt)
    J = sum((torch.tensor(w[n], device='cuda') * yy).sum() for n, yy in zip(NAMES, y))
    J.backward()
    rhs = sum(np.sum(v[n] * xx.grad.cpu().numpy()) for n, xx in zip(NAMES, x))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_gradient_matches_central_differences():
    st = small_jet(noisy=True)
    nsteps, remap_every, ckpt = 10, 5, 5
    dyn = Dycore(st)
    dyn.adj_enable()
    mask = gaussian_mask(st, 300e3, device='cuda')

    def theta(fields):
        return integrate(dyn, fields, nsteps, st.dt, remap_every, ckpt)[1] * P0K

    def loss(fields):
        return (mask * theta(fields) ** 2).sum()

    x = tensors(st)
    J = loss(x)
    J.backward()
    grad = torch.cat([xx.grad.flatten() for xx in x])
    gen = torch.Generator(device='cpu').manual_seed(5)
    worst = 0.
    for _ in range(4):
        d = torch.randn(grad.numel(), generator=gen, dtype=torch.float64).cuda()
        d /= d.norm()
        eps = 1e-6
        parts = torch.split(d, [xx.numel() for xx in x])
        with torch.no_grad():
            tp = theta([(xx + eps * p.view_as(xx)).detach() for xx, p in zip(x, parts)])
            tm = theta([(xx - eps * p.view_as(xx)).detach() for xx, p in zip(x, parts)])
            # J(x + eps d) - J(x - eps d) without cancelling two large sums
            fd = (mask * (tp - tm) * (tp + tm)).sum().item() / (2 * eps)
        ad = torch.dot(grad, d).item()
        worst = max(worst, abs(fd - ad) / abs(ad))
    assert worst <= 1e-4, worst


def test_differentiation_case_dot_product():
    """The 512 x 512 x 32 jet (seed 2), 20 steps, remap every 5, checkpoints
    every 5: <w, J v> from the tangent-linear oracle on all host cores
    against <J^T w, v> from the checkpointed CUDA adjoint."""
    import os
    st = ic.config(4)
    rng = np.random.default_rng(12)
    v = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    w = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    t = pyoracle.TLMModel(st, v, threads=len(os.sched_getaffinity(0)))
    for s in range(st.nsteps):
        t.cgrid_step(st.dt / 2)
        t.cgrid_halo()
        t.dgrid_step(st.dt)
        if (s + 1) % st.remap_every == 0:
            t.remap()
        t.dgrid_halo()
    lhs = sum(np.sum(w[n] * t.get(STATE[n])[1]) for n in NAMES)
    del t
    dyn = Dycore(st)
    dyn.adj_enable()
    x = tensors(st)
    y = integrate(dyn, x, st.nsteps, st.dt, st.remap_every, 5)
    J = sum((torch.tensor(w[n], device='cuda') * yy).sum() for n, yy in zip(NAMES, y))
    J.backward()
    rhs = sum(np.sum(v[n] * xx.grad.cpu().numpy()) for n, xx in zip(NAMES, x))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def _dot_product_case(st, nsteps, remap_every, ckpt, seed):
    rng = np.random.default_rng(seed)
    v = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    w = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    t = pyoracle.TLMModel(st, v, threads=8)
    for s in range(nsteps):
        t.cgrid_step(st.dt / 2)
        t.cgrid_halo()
        t.dgrid_step(st.dt)
        if (s + 1) % remap_every == 0:
            t.remap()
        t.dgrid_halo()
    lhs = sum(np.sum(w[n] * t.get(STATE[n])[1]) for n in NAMES)
    del t
    dyn = Dycore(st)
    dyn.adj_enable()
    x = tensors(st)
    y = integrate(dyn, x, nsteps, st.dt, remap_every, ckpt)
    J = sum((torch.tensor(w[n], device='cuda') * yy).sum() for n, yy in zip(NAMES, y))
    J.backward()
    rhs = sum(np.sum(v[n] * xx.grad.cpu().numpy()) for n, xx in zip(NAMES, x))
    dyn.close()
    return lhs, rhs


@pytest.mark.parametrize('member', [5, 7])
def test_ensemble_member_adjoint_dot_product(member):
    """Two members of the batched ensemble (seed 3) of different grid sizes
    and layer counts (64^2 x 48 and 128^2 x 64 jets), with their own time
    steps and remap interval: the gradient the ensemble leg computes for
    them (20 steps, checkpoints every 5) passes the dot-product test against
    the tangent-linear oracle."""
    st = ic.ensemble_members(8, seed=3)[member]
    assert (st.nx, st.nlay) == {5: (64, 48), 7: (128, 64)}[member]
    lhs, rhs = _dot_product_case(st, 20, st.remap_every, 5, seed=20 + member)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (st.name, lhs, rhs)


def test_gradient_run_to_run_spread():
    """The adjoint kernels add the adjoints of overlapping tile halos into
    global memory with atomics, so the order of those additions, and with it
    the last bits of the gradient, can change from run to run.  Two
    gradients of the same loss differ by at most 1e-12 of the gradient's
    norm (20 steps of the noisy jet, loss over every cell)."""
    st = small_jet(noisy=True)
    dyn = Dycore(st)
    dyn.adj_enable()
    grads = []
    for _ in range(2):
        x = tensors(st)
        y = integrate(dyn, x, 20, st.dt, 5, 5)
        ((y[1] * P0K) ** 2).sum().backward()
        grads.append(torch.cat([xx.grad.flatten() for xx in x]))
    dyn.close()
    spread = ((grads[0] - grads[1]).norm() / grads[0].norm()).item()
    print('relative run-to-run spread of the gradient: %.2e' % spread)
    assert spread <= 1e-12, spread
