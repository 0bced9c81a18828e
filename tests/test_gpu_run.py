"""The run driver from the reference's files: namelist + initial file ->
the CUDA library through the reference's time loop -> output.nc and the
restart file.  The final state equals stepping the same initial state
directly (bit for bit, with the radiation when the package has its
gas-optics tables), and each output record is the interval mean."""
import numpy as np
import pytest
from scipy.io import netcdf_file

from atmdyn import ic, Dycore, model, gas_optics
from atmdyn.io import write_initial, read_initial
from atmdyn.run import main

pytestmark = pytest.mark.gpu

NML = """&io_control
    initial_filename = 'init.nc'
    save_restart_file = T
    restart_filename = 'out/restart.nc'
/
&time_control
    max_timestep = "PT1M"
    run_duration = "PT10M"
    output_interval = "PT5M"
    radiation_interval = "PT3H"
    physics_interval = "PT5M"
    remap_interval = "PT4M"
/
&physics_parameters
    gravity = 9.807
    coriolis_parameter = 1e-4
    divergence_damping_coefficient = 0.15
    vorticity_damping_coefficient = 0.005
/
"""


def test_run_from_reference_files(tmp_path):
    st = ic.bubble_case(32, 24, 8, 50e3 * 4, 50e3 * 4, seed=5)
    write_initial(str(tmp_path / 'init.nc'), st)
    (tmp_path / 'config.nml').write_text(NML)
    out = str(tmp_path / 'out' / 'output.nc')
    summary = main([str(tmp_path / 'config.nml'), '--output', out, '--output-dtype', 'f8'])
    assert summary['stable'] and summary['steps'] == 10 and summary['remap_steps'] == [4, 8]
    assert len(summary['output_records']) == 2
    # the same run stepped directly
    st2 = read_initial(str(tmp_path / 'init.nc'))
    st2.gravity, st2.coriolis, st2.divdamp, st2.vortdamp = 9.807, 1e-4, 0.15, 0.005
    g = Dycore(st2)
    go = gas_optics.load_default()
    assert summary['radiation'] == (go is not None)
    if go is not None:
        g.set_radiation(go)
    means = []
    acc = {'dp': 0.}

    def on_step(n, time):
        acc['dp'] = acc['dp'] + 60.0 * g.get('dp')
        if n % 5 == 0:
            means.append(acc['dp'] / 300.0)
            acc['dp'] = 0.

    tc = model.TimeControl(dt_max=60.0, run_duration=600.0, dt_output=300.0, dt_radiation=10800.0,
                           dt_physics=300.0, dt_remap=240.0)
    r = model.run_model(g, tc, on_step=on_step, physics=True, radiation=go is not None)
    assert r.remap_steps == [4, 8]
    with netcdf_file(str(tmp_path / 'out' / 'restart.nc'), 'r', mmap=False) as nc:
        np.testing.assert_array_equal(nc.variables['dp'][:], g.get('dp'))
        np.testing.assert_array_equal(nc.variables['u'][:], g.get('ud'))
    with netcdf_file(out, 'r', mmap=False) as nc:
        assert nc.variables['dp'].shape == (2, 8, 24, 32)
        for rec in range(2):
            np.testing.assert_allclose(nc.variables['dp'][rec], means[rec], rtol=1e-15)
