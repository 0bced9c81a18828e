"""The reference's configuration and file formats on the host side.

* :func:`read_namelist` / :func:`read_config`: the three namelist groups of
  ``config.nml`` (src/mod_config.f90:34-99): ``io_control``,
  ``time_control`` (ISO-8601 durations) and ``physics_parameters``.
* :func:`parse_duration`: src/mod_util.f90:33-159, the reference's
  ISO-8601 duration reader (1 year = 365 d, 1 month = 30 d, first
  occurrence of each designator, M before the T is months, after it
  minutes).
* :func:`read_initial`: the initial-conditions file of
  src/mod_input.f90:21-228 (axes xc, yc, xf, yf, lay, lev, t; variables
  ak, bk, dp, pt, u, v, gzs, ts), dimensions mapped by name as the
  reference's reader does (src/mod_netcdf.f90:526-570), so the layout
  written by the reference's initial-condition generator and any
  permutation of it are accepted.
* :class:`OutputWriter` / :func:`write_restart`: output.nc and the restart
  file in the reference's layout (src/mod_output.f90:37-94, 176-230): a
  record dimension ``t``, FP32 data by default (``dtype='f8'`` keeps FP64).

netCDF-3 classic through ``scipy.io.netcdf_file`` (no netCDF library is
needed); netCDF-4/HDF5 files (xarray's default format) need the netCDF
library, which this image does not have.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np
from scipy.io import netcdf_file

from .ic import InitialState, cell_axes
from .model import TimeControl, NEVER


# ------------------------------------------------------------- namelist ----
def _strip_comment(line):
    out, q = [], None
    for ch in line:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in '\'"':
            q = ch
            out.append(ch)
        elif ch == '!':
            break
        else:
            out.append(ch)
    return ''.join(out)


def _value(tok):
    tok = tok.strip().rstrip(',').strip()
    if len(tok) >= 2 and tok[0] == tok[-1] and tok[0] in '\'"':
        return tok[1:-1]
    low = tok.lower()
    if low in ('t', '.true.', 'true', '.t.'):
        return True
    if low in ('f', '.false.', 'false', '.f.'):
        return False
    try:
        return int(tok)
    except ValueError:
        pass
    return float(low.replace('d', 'e'))


def read_namelist(text: str) -> dict:
    """{group: {key: value}} of a Fortran namelist text (scalars only)."""
    lines = [_strip_comment(l) for l in text.splitlines()]
    groups = {}
    cur = None
    for line in lines:
        s = line.strip()
        if not s:
            continue
        if s.startswith('&'):
            cur = s[1:].split()[0].lower()
            groups[cur] = {}
            s = s[1 + len(cur):].strip()
        if cur is None:
            continue
        end = s.endswith('/')
        if end:
            s = s[:-1]
        for m in re.finditer(r'(\w+)\s*=\s*(\'[^\']*\'|"[^"]*"|[^,\s]+)', s):
            groups[cur][m.group(1).lower()] = _value(m.group(2))
        if end:
            cur = None
    return groups


def parse_duration(s: str) -> float:
    """Seconds in an ISO-8601 duration, src/mod_util.f90:33-159."""
    s = s.strip()
    if not s.startswith('P'):
        raise ValueError('Could not read ISO8601 duration `%s`' % s)

    def scan(sub, ch):  # Fortran scan: 1-based position of the first ch, 0 if none
        i = sub.find(ch)
        return i + 1

    i_time = scan(s, 'T')
    if i_time > 0:
        head = s[:i_time]
        i_year, i_month, i_week, i_day = (scan(head, c) for c in 'YMWD')
        tail = s[i_time:]
        i_hour, i_minute, i_second = (scan(tail, c) for c in 'HMS')
        i_hour = i_time + i_hour if i_hour else 0
        i_minute = i_time + i_minute if i_minute else 0
        i_second = i_time + i_second if i_second else 0
    else:
        i_year, i_month, i_week, i_day = (scan(s, c) for c in 'YMWD')
        i_hour = i_minute = i_second = 0

    def read_real(a, b):  # s(a:b), 1-based inclusive
        txt = s[a - 1:b]
        try:
            v = float(txt)
        except ValueError:
            raise ValueError('Could not read ISO8601 duration `%s`' % s)
        if v < 0:
            raise ValueError('Could not read ISO8601 duration `%s`' % s)
        return v

    prev = 1
    n = dict(year=0., month=0., week=0., day=0., hour=0., minute=0., second=0.)
    for name, pos in (('year', i_year), ('month', i_month), ('week', i_week), ('day', i_day)):
        if pos:
            n[name] = read_real(prev + 1, pos - 1)
            prev = pos
    if i_time:
        prev = i_time
        for name, pos in (('hour', i_hour), ('minute', i_minute), ('second', i_second)):
            if pos:
                n[name] = read_real(prev + 1, pos - 1)
                prev = pos
    return (31536000. * n['year'] + 2592000. * n['month'] + 604800. * n['week'] + 86400. * n['day'] +
            3600. * n['hour'] + 60. * n['minute'] + 1. * n['second'])


@dataclass
class Config:
    """main_config of src/mod_config.f90:15-26 plus the physics constants."""
    initial_filename: str
    save_restart_file: bool
    restart_filename: str
    time: TimeControl
    gravity: float
    coriolis: float
    divdamp: float
    vortdamp: float
    extra: dict = field(default_factory=dict)


def read_config(path_or_text: str) -> Config:
    """read_config_file (src/mod_config.f90:27-99)."""
    text = path_or_text
    if '&' not in path_or_text:
        with open(path_or_text) as f:
            text = f.read()
    g = read_namelist(text)
    for grp in ('io_control', 'time_control', 'physics_parameters'):
        if grp not in g:
            raise ValueError('Could not read `%s` namelist' % grp)
    io, tc, ph = g['io_control'], g['time_control'], g['physics_parameters']

    def dur(key):
        return parse_duration(tc[key]) if key in tc else NEVER

    t = TimeControl(dt_max=dur('max_timestep'), run_duration=dur('run_duration'),
                    dt_output=dur('output_interval'), dt_radiation=dur('radiation_interval'),
                    dt_physics=dur('physics_interval'), dt_remap=dur('remap_interval'))
    return Config(initial_filename=io.get('initial_filename', 'initial.nc'),
                  save_restart_file=bool(io.get('save_restart_file', False)),
                  restart_filename=io.get('restart_filename', 'restart.nc'), time=t,
                  gravity=float(ph['gravity']), coriolis=float(ph['coriolis_parameter']),
                  divdamp=float(ph['divergence_damping_coefficient']),
                  vortdamp=float(ph['vorticity_damping_coefficient']))


# --------------------------------------------------------------- netCDF ----
def _by_name(var, want, tname='t'):
    """The variable's data as an array over the dimensions ``want`` (one of
    alternatives per position, e.g. (('lay',), ('yc', 'yf'), ('xc', 'xf')))
    taking the first record of ``t``."""
    dims = list(var.dimensions)
    data = np.asarray(var[:])
    if tname in dims:
        data = np.take(data, 0, axis=dims.index(tname))
        dims.remove(tname)
    order = []
    for alts in want:
        hit = [d for d in dims if d in alts]
        if len(hit) != 1:
            raise ValueError('variable with dimensions %s lacks one of %s' % (var.dimensions, alts))
        order.append(dims.index(hit[0]))
    return np.ascontiguousarray(np.transpose(data, order), dtype=np.float64)


def read_initial(path: str, config: Config | None = None) -> InitialState:
    """read_initial_file + init_prognostic_fields (src/mod_input.f90:21-228)."""
    with netcdf_file(path, 'r', mmap=False) as nc:
        for name in ('xc', 'yc', 'xf', 'yf', 'lay', 'lev'):
            if name not in nc.dimensions:
                raise ValueError('Could not find axis `%s` in initial condition netCDF.' % name)
        nx, ny, nlay = nc.dimensions['xc'], nc.dimensions['yc'], nc.dimensions['lay']
        if nc.dimensions['xf'] != nx or nc.dimensions['yf'] != ny:
            raise ValueError('Inconsistent horizontal axis sizes in initial condition netCDF.')
        if nc.dimensions['lev'] != nlay + 1:
            raise ValueError('Inconsistent vertical axis sizes in initial condition netCDF.')
        xc = np.asarray(nc.variables['xc'][:], dtype=np.float64)
        yc = np.asarray(nc.variables['yc'][:], dtype=np.float64)
        dx, dy = xc[1] - xc[0], yc[1] - yc[0]
        tol = 1e-3
        if not np.all(np.abs(np.diff(xc)) - abs(dx) < tol) or not np.all(np.abs(np.diff(yc)) - abs(dy) < tol):
            raise ValueError('Spacing of coordinate points in initial condition netCDF is not uniform.')
        t0 = float(np.asarray(nc.variables['t'][:])[0]) if 't' in nc.variables else 0.0
        ak = np.asarray(nc.variables['ak'][:], dtype=np.float64)
        bk = np.asarray(nc.variables['bk'][:], dtype=np.float64)
        lay, y, x = ('lay',), ('yc', 'yf'), ('xc', 'xf')
        f = {n: _by_name(nc.variables[n], (lay, y, x)) for n in ('dp', 'pt', 'u', 'v')}
        gzs = _by_name(nc.variables['gzs'], (y, x))
        ts = _by_name(nc.variables['ts'], (y, x)) if 'ts' in nc.variables else None
    st = InitialState(nx, ny, nlay, float(dx), float(dy), ak, bk, f['dp'], f['pt'], f['u'], f['v'], gzs)
    st.t_initial = t0
    st.ts = ts
    st.xc, st.yc = xc, yc  # the radiation's cell radius (src/mod_input.f90:233-243)
    if config is not None:
        st.gravity, st.coriolis = config.gravity, config.coriolis
        st.divdamp, st.vortdamp = config.divdamp, config.vortdamp
    return st


def write_initial(path: str, st: InitialState, ts=None, t0: float = 0.0):
    """An initial-conditions file with the variables and dimension order of
    the reference's generator (variables over (yc, xc, lay, t)).  netCDF-3
    allows a record dimension only in first place, so ``t`` is a fixed
    dimension of length 1 here; the reference reads it by name either way."""
    with netcdf_file(path, 'w') as nc:
        nc.createDimension('t', 1)
        for n, size in (('xc', st.nx), ('yc', st.ny), ('xf', st.nx), ('yf', st.ny), ('lay', st.nlay),
                        ('lev', st.nlay + 1)):
            nc.createDimension(n, size)
        xc, yc = cell_axes(st)  # the generator's axes (scripts/ic_generator.py:20-24)
        axes = {'xc': xc, 'xf': xc - st.dx / 2, 'yc': yc, 'yf': yc - st.dy / 2,
                'lay': np.arange(1, st.nlay + 1), 'lev': np.arange(1, st.nlay + 2)}
        for n, v in axes.items():
            nc.createVariable(n, 'f8', (n,))[:] = v
        tv = nc.createVariable('t', 'f8', ('t',))
        tv[0] = t0
        for n, a, d in (('dp', st.dp, ('yc', 'xc', 'lay', 't')), ('pt', st.pt, ('yc', 'xc', 'lay', 't')),
                        ('u', st.u, ('yc', 'xf', 'lay', 't')), ('v', st.v, ('yf', 'xc', 'lay', 't'))):
            nc.createVariable(n, 'f8', d)[:] = np.transpose(a, (1, 2, 0))[..., None]
        nc.createVariable('gzs', 'f8', ('yc', 'xc', 't'))[:] = np.asarray(st.gzs)[..., None]
        tsv = np.full((st.ny, st.nx), 288.0) if ts is None else ts
        nc.createVariable('ts', 'f8', ('yc', 'xc', 't'))[:] = tsv[..., None]
        nc.createVariable('ak', 'f8', ('lev',))[:] = st.ak
        nc.createVariable('bk', 'f8', ('lev',))[:] = st.bk


class OutputWriter:
    """output.nc of src/mod_output.f90:37-94,144-176: axes t (record), x, y,
    lay, lev; interval means of dp, pt, u, v over (t, lay, y, x), ts over
    (t, y, x), nflx over (t, lev, y, x)."""

    def __init__(self, path: str, st: InitialState, dtype: str = 'f4'):
        self.nc = netcdf_file(path, 'w')
        nc = self.nc
        Lx, Ly = st.nx * st.dx, st.ny * st.dy
        nc.createDimension('t', None)
        for n, size in (('x', st.nx), ('y', st.ny), ('lay', st.nlay), ('lev', st.nlay + 1)):
            nc.createDimension(n, size)
        nc.createVariable('t', 'f8', ('t',))
        nc.createVariable('x', 'f8', ('x',))[:] = -.5 * Lx + (np.arange(st.nx) + .5) * st.dx
        nc.createVariable('y', 'f8', ('y',))[:] = -.5 * Ly + (np.arange(st.ny) + .5) * st.dy
        nc.createVariable('lay', 'f8', ('lay',))[:] = np.arange(1, st.nlay + 1)
        nc.createVariable('lev', 'f8', ('lev',))[:] = np.arange(1, st.nlay + 2)
        for n in ('dp', 'pt', 'u', 'v'):
            nc.createVariable(n, dtype, ('t', 'lay', 'y', 'x'))
        nc.createVariable('ts', dtype, ('t', 'y', 'x'))
        nc.createVariable('nflx', dtype, ('t', 'lev', 'y', 'x'))
        self.n = 0

    def write(self, time: float, means: dict):
        """One record: ``means`` maps dp, pt, u, v, nflx (and optionally ts)
        to interval means shaped (K, ny, nx) ((ny, nx) for ts)."""
        nc = self.nc
        nc.variables['t'][self.n] = time
        for n in ('dp', 'pt', 'u', 'v', 'nflx'):
            nc.variables[n][self.n] = means[n]
        if 'ts' in means:
            nc.variables['ts'][self.n] = means['ts']
        self.n += 1
        nc.flush()

    def close(self):
        self.nc.close()


def write_restart(path: str, st: InitialState, fields: dict, time: float, ts=None, dtype: str = 'f4'):
    """write_restart_file (src/mod_output.f90:178-230): dp, pt on (lay, yc,
    xc), u on (lay, yf... as the reference's staggering), gzs, ts."""
    with netcdf_file(path, 'w') as nc:
        nc.createDimension('t', None)
        Lx, Ly = st.nx * st.dx, st.ny * st.dy
        for n, size in (('xc', st.nx), ('xf', st.nx), ('yc', st.ny), ('yf', st.ny), ('lay', st.nlay)):
            nc.createDimension(n, size)
        nc.createVariable('t', 'f8', ('t',))[0] = time
        nc.createVariable('xc', 'f8', ('xc',))[:] = -.5 * Lx + (np.arange(st.nx) + .5) * st.dx
        nc.createVariable('xf', 'f8', ('xf',))[:] = -.5 * Lx + np.arange(st.nx) * st.dx
        nc.createVariable('yc', 'f8', ('yc',))[:] = -.5 * Ly + (np.arange(st.ny) + .5) * st.dy
        nc.createVariable('yf', 'f8', ('yf',))[:] = -.5 * Ly + np.arange(st.ny) * st.dy
        nc.createVariable('lay', 'f8', ('lay',))[:] = np.arange(1, st.nlay + 1)
        nc.createVariable('dp', dtype, ('lay', 'yc', 'xc'))[:] = fields['dp']
        nc.createVariable('pt', dtype, ('lay', 'yc', 'xc'))[:] = fields['pt']
        nc.createVariable('u', dtype, ('lay', 'yf', 'xc'))[:] = fields['ud']
        nc.createVariable('v', dtype, ('lay', 'yc', 'xf'))[:] = fields['vd']
        nc.createVariable('gzs', dtype, ('yc', 'xc'))[:] = st.gzs
        nc.createVariable('ts', dtype, ('yc', 'xc'))[:] = np.full((st.ny, st.nx), 288.0) if ts is None else ts
