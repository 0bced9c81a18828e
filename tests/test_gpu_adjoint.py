"""Adjoint of the FP64 step on the GPU against the oracle's tangent-linear model.

Dot-product tests: for random tangents v of a stage's inputs (the CPU
tangent-linear oracle, branches frozen at the FP64 trajectory) and random
adjoints w of its outputs (the CUDA adjoint kernels), <w, J v> and
<J^T w, v> agree to 1e-12 relative.  The base state is a bubble with
noise on every field, so that no limiter sits exactly on a tie (a tie is a
kink where the one-sided derivatives differ).
"""
import copy

import numpy as np
import pytest

from atmdyn import ic, Dycore
import pyoracle

pytestmark = pytest.mark.gpu

H = 7
TOL = 1e-12
NAMES = ('dp', 'pt', 'ud', 'vd')
STATE = {'dp': pyoracle.DP, 'pt': pyoracle.PT, 'ud': pyoracle.UD, 'vd': pyoracle.VD}
CGRID = {'dpc': pyoracle.DPC, 'ptc': pyoracle.PTC, 'uc': pyoracle.UC, 'vc': pyoracle.VC}
SCALE = {'dp': 10.0, 'pt': 0.01, 'ud': 0.5, 'vd': 0.5, 'dpc': 10.0, 'ptc': 0.01, 'uc': 0.5, 'vc': 0.5}


def generic_state(nx=40, ny=24, nlay=6, seed=0):
    st = ic.bubble_case(nx, ny, nlay, 200e3, 200e3, radius=800e3, u0=12.0)
    rng = np.random.default_rng(seed)
    st.v = st.v + 2.0
    st.dp = st.dp + rng.normal(0, 5.0, st.dp.shape)
    st.pt = st.pt * (1 + rng.normal(0, 1e-3, st.pt.shape))
    st.u = st.u + rng.normal(0, 0.5, st.u.shape)
    st.v = st.v + rng.normal(0, 0.5, st.v.shape)
    return st


def padded_shape(st):
    return (st.nlay, st.ny + 2 * H, st.nx + 2 * H)


def rand(rng, st, name):
    return rng.normal(0, SCALE[name], padded_shape(st))


def mask(st, r):
    m = np.zeros(padded_shape(st))
    m[:, H - r:H + st.ny + r, H - r:H + st.nx + r] = 1.
    return m


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def tlm_from_gpu(g, st, tangents):
    """A tangent-linear oracle whose state values are the GPU's padded fields."""
    t = pyoracle.TLMModel(st)
    for n in NAMES:
        t.set(STATE[n], g.get(n, halo=True), tangents.get(n), halo=True)
    return t


def test_cgrid_step_dot_product():
    st = generic_state()
    rng = np.random.default_rng(1)
    g = Dycore(st)
    g.adj_enable()
    v = {n: rand(rng, st, n) for n in NAMES}
    t = tlm_from_gpu(g, st, v)
    t.cgrid_step(st.dt / 2)
    w = {n: rand(rng, st, n) * mask(st, 2 if n in ('dpc', 'ptc') else 0) for n in CGRID}
    lhs = sum(np.sum(w[n] * t.get(CGRID[n], halo=True)[1]) for n in CGRID)
    for n in CGRID:
        g.adj_set('in', n, w[n])
    g.adj_cgrid_step(st.dt / 2)
    rhs = sum(np.sum(v[n] * g.adj_get('in', n)) for n in NAMES)
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


def test_dgrid_step_dot_product():
    st = generic_state(seed=2)
    rng = np.random.default_rng(3)
    g = Dycore(st)
    g.adj_enable()
    vs = {n: rand(rng, st, n) for n in NAMES}
    t = tlm_from_gpu(g, st, vs)
    t.cgrid_step(st.dt / 2)
    t.cgrid_halo()
    vc = {n: rand(rng, st, n) for n in CGRID}
    for n in CGRID:
        t.set(CGRID[n], t.get(CGRID[n], halo=True)[0], vc[n], halo=True)
    t.dgrid_step(st.dt)
    w = {n: rand(rng, st, n) for n in NAMES}
    lhs = sum(np.sum(w[n] * t.get(STATE[n], halo=True)[1]) for n in NAMES)
    for n in NAMES:
        g.adj_set('out', n, w[n])
    g.adj_dgrid_step(st.dt)
    rhs = sum(np.sum(vs[n] * g.adj_get('in', n)) for n in NAMES)
    rhs += sum(np.sum(vc[n] * g.adj_get('in', n)) for n in CGRID)
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


def test_remap_dot_product():
    st = generic_state(seed=4)
    rng = np.random.default_rng(5)
    g = Dycore(st)
    g.adj_enable()
    g.cgrid_step(st.dt / 2)
    g.cgrid_halo()
    g.dgrid_step(st.dt)  # the pre-remap state, with last step's ring on the winds
    v = {n: rand(rng, st, n) for n in NAMES}
    t = tlm_from_gpu(g, st, v)
    t.remap()
    w = {n: rand(rng, st, n) for n in NAMES}
    lhs = sum(np.sum(w[n] * t.get(STATE[n], halo=True)[1]) for n in NAMES)
    for n in NAMES:
        g.adj_set('out', n, w[n])
    g.adj_remap()
    rhs = sum(np.sum(v[n] * g.adj_get('in', n)) for n in NAMES)
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


def test_remap_dot_product_non_monotone_columns():
    """Columns whose source pressure is not monotone (one layer of negative
    thickness) take the all-pairs path of the remap and of its adjoint."""
    st = generic_state(seed=6)
    for j, i in ((3, 5), (10, 20), (17, 31)):
        st.dp[2, j, i] = -0.3 * st.dp[2, j, i]
    rng = np.random.default_rng(7)
    g = Dycore(st)
    g.adj_enable()
    v = {n: rand(rng, st, n) for n in NAMES}
    t = tlm_from_gpu(g, st, v)
    t.remap()
    w = {n: rand(rng, st, n) for n in NAMES}
    lhs = sum(np.sum(w[n] * t.get(STATE[n], halo=True)[1]) for n in NAMES)
    for n in NAMES:
        g.adj_set('out', n, w[n])
    g.adj_remap()
    rhs = sum(np.sum(v[n] * g.adj_get('in', n)) for n in NAMES)
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


def test_halo_dot_products():
    st = generic_state(seed=6)
    rng = np.random.default_rng(7)
    g = Dycore(st)
    g.adj_enable()
    v = {n: rand(rng, st, n) for n in NAMES}
    t = tlm_from_gpu(g, st, v)
    t.dgrid_halo()
    w = {n: rand(rng, st, n) for n in NAMES}
    lhs = sum(np.sum(w[n] * t.get(STATE[n], halo=True)[1]) for n in NAMES)
    for n in NAMES:
        g.adj_set('out', n, w[n])
    g.adj_halo('out')
    rhs = sum(np.sum(v[n] * g.adj_get('out', n)) for n in NAMES)
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)
    # the C-grid fields
    t.cgrid_step(st.dt / 2)
    vc = {n: rand(rng, st, n) for n in CGRID}
    for n in CGRID:
        t.set(CGRID[n], t.get(CGRID[n], halo=True)[0], vc[n], halo=True)
    t.cgrid_halo()
    wc = {n: rand(rng, st, n) for n in CGRID}
    lhs = sum(np.sum(wc[n] * t.get(CGRID[n], halo=True)[1]) for n in CGRID)
    for n in CGRID:
        g.adj_set('in', n, wc[n])
    g.adj_cgrid_halo()
    rhs = sum(np.sum(vc[n] * g.adj_get('in', n)) for n in CGRID)
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)


@pytest.mark.parametrize('remap_every', [2, 100])
def test_three_steps_dot_product(remap_every):
    """Three whole steps (C, halo, D, [remap], halo) through atm_adj_step."""
    st = generic_state(32, 24, 6, seed=8)
    rng = np.random.default_rng(9)
    nsteps = 3
    v = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    t = pyoracle.TLMModel(st, v)
    for s in range(nsteps):
        t.cgrid_step(st.dt / 2)
        t.cgrid_halo()
        t.dgrid_step(st.dt)
        if (s + 1) % remap_every == 0:
            t.remap()
        t.dgrid_halo()
    w = {n: rng.normal(0, SCALE[n], (st.nlay, st.ny, st.nx)) for n in NAMES}
    lhs = sum(np.sum(w[n] * t.get(STATE[n])[1]) for n in NAMES)
    lam = {n: np.pad(w[n], ((0, 0), (H, H), (H, H))) for n in NAMES}
    for s in reversed(range(nsteps)):
        g = Dycore(st)
        for q in range(s):
            g.step(st.dt, remap=(q + 1) % remap_every == 0, check_stable=False)
        g.adj_enable()
        for n in NAMES:
            g.adj_set('out', n, lam[n])
        g.adj_step(st.dt, remap=(s + 1) % remap_every == 0)
        lam = {n: g.adj_get('out', n) for n in NAMES}
        if s == 0:
            g.adj_halo('out')
            lam = {n: g.adj_get('out', n, halo=False) for n in NAMES}
        g.close()
    rhs = sum(np.sum(v[n] * lam[n]) for n in NAMES)
    assert rel(lhs, rhs) <= TOL, (lhs, rhs)
