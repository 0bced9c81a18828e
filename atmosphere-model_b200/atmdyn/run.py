"""Run the dynamical core from the reference's own files.

    python -m atmdyn.run [config.nml] [--precision fp64|mixed] [--output output/output.nc]
                         [--max-steps N] [--output-dtype f4|f8] [--gas-optics tables.npz | --no-radiation]

Reads the namelist (src/mod_config.f90:27-99) and the initial-conditions
file it names (src/mod_input.f90:21-228), steps the CUDA library through
the reference's time loop (src/mod_model.f90:112-199: schedule, C/D-grid
steps, remap when due, halo fills, stability check), accumulates the
output means on the device (src/mod_output.f90:94-142) and writes them to
output.nc when an output interval ends, and writes the restart file at the
end when the namelist asks for it.  The physics (src/mod_physics.f90: dry
convective adjustment, surface heating) and the radiation
(src/mod_radiation.f90: two-stream shortwave and longwave over 16 g-points)
run on the device when due.  The radiation needs the gas-optics tables
(:mod:`atmdyn.gas_optics`): ``--gas-optics`` names an ``.npz``, else the
package's default tables are used; without tables (or with
``--no-radiation``) the net flux stays zero.
"""
from __future__ import annotations

import argparse
import json
import os

from . import gas_optics
from .dycore import Dycore
from .io import read_config, read_initial, OutputWriter, write_restart
from .model import run_model, TimeControl


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('config', nargs='?', default='config.nml')
    ap.add_argument('--precision', default='fp64', choices=['fp64', 'mixed'])
    ap.add_argument('--output', default='output/output.nc')
    ap.add_argument('--output-dtype', default='f4', choices=['f4', 'f8'])
    ap.add_argument('--max-steps', type=int, default=None)
    ap.add_argument('--gas-optics', default=None, help='gas-optics tables (.npz, atmdyn.gas_optics.save)')
    ap.add_argument('--no-radiation', action='store_true')
    args = ap.parse_args(argv)
    cfg = read_config(args.config)
    base = os.path.dirname(os.path.abspath(args.config))
    init = cfg.initial_filename if os.path.isabs(cfg.initial_filename) else os.path.join(base, cfg.initial_filename)
    st = read_initial(init, cfg)
    t = cfg.time
    tc = TimeControl(dt_max=t.dt_max, run_duration=t.run_duration, dt_output=t.dt_output,
                     dt_radiation=t.dt_radiation, dt_physics=t.dt_physics, dt_remap=t.dt_remap,
                     t_initial=st.t_initial)
    dyn = Dycore(st, args.precision)
    go = None
    if not args.no_radiation:
        go = gas_optics.load(args.gas_optics) if args.gas_optics else gas_optics.load_default()
    if go is not None:
        dyn.set_radiation(go)
    dyn.output_enable()
    os.makedirs(os.path.dirname(os.path.abspath(args.output)), exist_ok=True)
    writer = OutputWriter(args.output, st, dtype=args.output_dtype)
    records = []

    def write(stamp):
        means = {n: dyn.output_read(n) for n in ('dp', 'pt', 'u', 'v', 'nflx')}
        if st.ts is not None:
            means['ts'] = dyn.output_read('ts')[0]
        writer.write(stamp, means)
        dyn.output_reset()
        records.append(stamp)

    res = run_model(dyn, tc, max_steps=args.max_steps, accumulate=dyn.accumulate_output, write=write,
                    physics=True, radiation=go is not None)
    writer.close()
    restart = None
    if cfg.save_restart_file and res.stable:
        restart = cfg.restart_filename if os.path.isabs(cfg.restart_filename) else os.path.join(
            base, cfg.restart_filename)
        os.makedirs(os.path.dirname(os.path.abspath(restart)), exist_ok=True)
        ts = dyn.get('ts')[0] if st.ts is not None else None
        write_restart(restart, st, dyn.state(), res.time, ts=ts, dtype=args.output_dtype)
    summary = {'steps': res.steps, 'time': res.time, 'stable': res.stable, 'remap_steps': res.remap_steps,
               'output_records': records, 'output': args.output, 'restart': restart,
               'radiation': go is not None}
    print(json.dumps(summary))
    dyn.close()
    return summary


if __name__ == '__main__':
    main()
