"""On-device output accumulation against a restatement of the reference's
accumulate_output / write_output (src/mod_output.f90:94-176) on the host:
the same FP64 operations in the same order, so the means agree bit for bit."""
import numpy as np
import pytest

from atmdyn import ic, Dycore, model

pytestmark = pytest.mark.gpu


def test_accumulated_means_bit_exact():
    st = ic.bubble_case(40, 24, 8, 200e3, 200e3, radius=800e3)
    g = Dycore(st)
    g.output_enable()
    H = 7
    sums = {n: 0. for n in ('dp', 'pt', 'u', 'v')}
    t = 0.
    for s in range(6):
        g.step(st.dt, remap=(s + 1) % 5 == 0)
        g.accumulate_output(st.dt)
        dp, pt = g.get('dp'), g.get('pt')
        ud, vd = g.get('ud', halo=True), g.get('vd', halo=True)
        ny, nx = st.ny, st.nx
        u = st.dt * .5 * (ud[:, H:H + ny, H:H + nx] + ud[:, H + 1:H + ny + 1, H:H + nx])
        v = st.dt * .5 * (vd[:, H:H + ny, H:H + nx] + vd[:, H:H + ny, H + 1:H + nx + 1])
        sums['dp'] = sums['dp'] + st.dt * dp
        sums['pt'] = sums['pt'] + st.dt * pt
        sums['u'] = sums['u'] + u
        sums['v'] = sums['v'] + v
        t = t + st.dt
    for n in ('dp', 'pt', 'u', 'v'):
        np.testing.assert_array_equal(g.output_read(n), sums[n] / t)
    np.testing.assert_array_equal(g.output_read('nflx'), np.zeros((st.nlay + 1, st.ny, st.nx)))
    g.output_reset()
    g.step(st.dt)
    g.accumulate_output(2.0)
    np.testing.assert_array_equal(g.output_read('dp'), (2.0 * g.get('dp')) / 2.0)
