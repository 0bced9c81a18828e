"""The reference's namelist, ISO-8601 durations and netCDF layouts on the
host (src/mod_config.f90:27-99, src/mod_util.f90:33-159,
src/mod_input.f90:21-228, src/mod_output.f90:37-230)."""
import numpy as np
import pytest
from scipy.io import netcdf_file

from atmdyn import ic
from atmdyn.io import parse_duration, read_namelist, read_config, write_initial, read_initial, OutputWriter

NML = """
&io_control
    initial_filename = 'start.nc'   ! a comment
    save_restart_file = T
    restart_filename = "out/rst.nc"
/

&time_control
    max_timestep = "PT90S"
    run_duration = "P1DT6H"
    output_interval = "PT30M"
    radiation_interval = "PT3H"
    physics_interval = "PT5M"
    remap_interval = "PT15M"
/

&physics_parameters
    gravity = 9.81
    coriolis_parameter = 2d-4
    divergence_damping_coefficient = 0.1,
    vorticity_damping_coefficient = 0.004
/
"""


@pytest.mark.parametrize('s, sec', [('PT2M', 120.), ('P5D', 432000.), ('PT1H', 3600.), ('PT3H', 10800.),
                                    ('P1Y2M3W4DT5H6M7S', 31536000. + 2 * 2592000. + 3 * 604800. + 4 * 86400. +
                                     5 * 3600. + 6 * 60. + 7.),
                                    ('P1M', 2592000.), ('PT1M', 60.), ('PT0.5S', .5), ('P1DT12H', 129600.)])
def test_parse_duration(s, sec):
    assert parse_duration(s) == sec


def test_parse_duration_rejects():
    for bad in ('T1H', '1D', 'PXD'):
        with pytest.raises(ValueError):
            parse_duration(bad)


def test_namelist_and_config():
    g = read_namelist(NML)
    assert g['io_control']['save_restart_file'] is True
    assert g['io_control']['restart_filename'] == 'out/rst.nc'
    c = read_config(NML)
    assert c.initial_filename == 'start.nc'
    assert c.time.dt_max == 90. and c.time.run_duration == 86400. + 6 * 3600.
    assert c.time.dt_output == 1800. and c.time.dt_remap == 900.
    assert (c.gravity, c.coriolis, c.divdamp, c.vortdamp) == (9.81, 2e-4, 0.1, 0.004)


def test_initial_file_round_trip(tmp_path):
    st = ic.bubble_case(12, 10, 5, 50e3, 50e3, seed=3)
    p = str(tmp_path / 'init.nc')
    write_initial(p, st, t0=120.0)
    r = read_initial(p)
    assert (r.nx, r.ny, r.nlay, r.dx, r.dy, r.t_initial) == (12, 10, 5, 50e3, 50e3, 120.0)
    for a, b in ((r.dp, st.dp), (r.pt, st.pt), (r.u, st.u), (r.v, st.v), (r.gzs, st.gzs), (r.ak, st.ak)):
        np.testing.assert_array_equal(a, b)


def test_output_writer(tmp_path):
    st = ic.bubble_case(8, 6, 4, 50e3, 50e3)
    p = str(tmp_path / 'out.nc')
    w = OutputWriter(p, st, dtype='f8')
    for t in (3600., 7200.):
        w.write(t, {'dp': st.dp * t, 'pt': st.pt, 'u': st.u, 'v': st.v, 'nflx': np.zeros((5, 6, 8))})
    w.close()
    with netcdf_file(p, 'r', mmap=False) as nc:
        assert nc.variables['dp'].dimensions == ('t', 'lay', 'y', 'x')
        np.testing.assert_array_equal(nc.variables['t'][:], [3600., 7200.])
        np.testing.assert_array_equal(nc.variables['dp'][1], st.dp * 7200.)
