"""Gas-optics tables of the radiation scheme (src/mod_gas_optics.f90,
src/mod_solar.f90).

The reference compiles its correlated-k tables into the model as Fortran
parameter arrays: 16 g-points; shortwave and longwave absorption
coefficients on 53 pressures x 6 temperatures (the temperature grid moves
with pressure); a Rayleigh scattering coefficient per g-point; Planck
functions on 231 temperatures; and the fraction of the solar irradiance
each g-point carries.  Those numbers are data, not code of this library:
:func:`from_fortran` reads them out of the reference's own source files
(the user's checkout), :func:`save` / :func:`load` keep them as an ``.npz``,
and the CUDA library receives them through ``atm_set_gas_optics``.  The
literals in those files carry no kind suffix, so Fortran reads them as
default (single-precision) reals and widens them to FP64; :func:`from_fortran`
rounds them the same way, so the arrays hold exactly the reference's values.

:func:`synthetic` builds tables of the same shapes from a seed (absorption
growing with pressure and temperature, Planck functions from Planck's law on
16 bands), for tests that need no reference files.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, fields

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PATH = os.path.join(HERE, '_tables', 'ecckd_climate16.npz')

# the reference's fixed radiation parameters (src/mod_radiation.f90:107-109;
# .3 and .99 are default-real literals)
SOLAR_ZENITH_ANGLE = 0.0
SURFACE_ALBEDO = float(np.float32(.3))
SURFACE_EMISSIVITY = float(np.float32(.99))


@dataclass
class GasOptics:
    """Arrays in the reference's Fortran index order, flattened C-order from
    the last Fortran index: ``temperatures[p, t]`` is ``temperatures(t, p)``,
    ``sw_absorption[g, p, t]`` is ``shortwave_absorption_lut(t, p, g)`` and
    ``planck[g, t]`` is ``planckian_lut(t, g)``."""
    pressures: np.ndarray            # (n_p,) ascending, Pa
    temperatures: np.ndarray         # (n_p, n_t) ascending in t, K
    sw_absorption: np.ndarray        # (n_g, n_p, n_t) m2/kg
    sw_scattering: np.ndarray        # (n_g,) m2/kg (Rayleigh)
    lw_absorption: np.ndarray        # (n_g, n_p, n_t) m2/kg
    planck_temperatures: np.ndarray  # (n_planck,) ascending, K
    planck: np.ndarray               # (n_g, n_planck) W/m2/sr
    irradiance_fraction: np.ndarray  # (n_g,)

    @property
    def n_g(self) -> int:
        return int(self.sw_scattering.shape[0])

    def validate(self) -> 'GasOptics':
        ng = self.n_g
        npr, nt = self.temperatures.shape
        npl = self.planck_temperatures.shape[0]
        want = {'pressures': (npr,), 'temperatures': (npr, nt), 'sw_absorption': (ng, npr, nt),
                'sw_scattering': (ng,), 'lw_absorption': (ng, npr, nt), 'planck_temperatures': (npl,),
                'planck': (ng, npl), 'irradiance_fraction': (ng,)}
        for f in fields(self):
            a = np.ascontiguousarray(getattr(self, f.name), dtype=np.float64)
            if a.shape != want[f.name]:
                raise ValueError('%s has shape %s, expected %s' % (f.name, a.shape, want[f.name]))
            setattr(self, f.name, a)
        if npr < 2 or nt < 2 or npl < 2:
            raise ValueError('each lookup axis needs at least two points')
        if not (np.all(np.diff(self.pressures) > 0) and np.all(np.diff(self.temperatures, axis=1) > 0)
                and np.all(np.diff(self.planck_temperatures) > 0)):
            raise ValueError('lookup axes must be strictly ascending')
        return self


# ---- the reference's source files ---------------------------------------------------------

# arrays of mod_gas_optics.f90 / mod_solar.f90 and the field each one fills
_NAMES = {'pressures': 'pressures', 'temperatures': 'temperatures',
          'shortwave_absorption_lut': 'sw_absorption', 'rayleigh_scattering_lut': 'sw_scattering',
          'longwave_absorption_lut': 'lw_absorption', 'planckian_temperatures': 'planck_temperatures',
          'planckian_lut': 'planck', 'irradiance_fraction': 'irradiance_fraction'}
_NUM = re.compile(r'[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eEdD][-+]?\d+)?(?:_\w+)?')


def _literal(tok: str) -> float:
    """A Fortran real literal: a ``d`` exponent or a kind suffix makes it
    double precision; otherwise it is a default (single-precision) real."""
    double = '_' in tok or 'd' in tok.lower()
    v = float(tok.split('_')[0].lower().replace('d', 'e'))
    return v if double else float(np.float32(v))


def _arrays(text: str) -> dict:
    text = '\n'.join(line.split('!', 1)[0] for line in text.splitlines())
    out = {}
    for m in re.finditer(r'\b(\w+)\s*\(([^()]*)\)\s*(?:&\s*)?=\s*(?:&\s*)?(reshape\s*\(\s*(?:&\s*)?)?\[', text):
        name = m.group(1)
        if name not in _NAMES:
            continue
        end = text.index(']', m.end())
        out[name] = np.array([_literal(t) for t in _NUM.findall(text[m.end():end].replace('&', ' '))])
    return out


def from_fortran(gas_optics_f90: str, solar_f90: str) -> GasOptics:
    """Read the tables out of the reference's mod_gas_optics.f90 and
    mod_solar.f90 (the parameter arrays of mod_gas_optics.f90:25-132,
    143-1841, 1852-1857, 1870-3568, 3579-4549 and mod_solar.f90:16-23)."""
    with open(gas_optics_f90) as f:
        go_text = f.read()
    with open(solar_f90) as f:
        solar_text = f.read()
    return from_fortran_text(go_text, solar_text)


def from_fortran_text(gas_optics_src: str, solar_src: str) -> GasOptics:
    """:func:`from_fortran` on the two files' contents."""
    a = _arrays(gas_optics_src)
    a.update(_arrays(solar_src))
    missing = [n for n in _NAMES if n not in a]
    if missing:
        raise ValueError('arrays not found: %s' % ', '.join(missing))
    ng = a['rayleigh_scattering_lut'].size
    npr = a['pressures'].size
    nt = a['temperatures'].size // npr
    npl = a['planckian_temperatures'].size
    # Fortran order (t, p[, g]) -> C order [g][p][t]
    return GasOptics(pressures=a['pressures'],
                     temperatures=a['temperatures'].reshape(npr, nt),
                     sw_absorption=a['shortwave_absorption_lut'].reshape(ng, npr, nt),
                     sw_scattering=a['rayleigh_scattering_lut'],
                     lw_absorption=a['longwave_absorption_lut'].reshape(ng, npr, nt),
                     planck_temperatures=a['planckian_temperatures'],
                     planck=a['planckian_lut'].reshape(ng, npl),
                     irradiance_fraction=a['irradiance_fraction']).validate()


def from_reference_tree(root: str) -> GasOptics:
    """:func:`from_fortran` on ``root``/src of a reference checkout."""
    return from_fortran(os.path.join(root, 'src', 'mod_gas_optics.f90'), os.path.join(root, 'src', 'mod_solar.f90'))


def save(go: GasOptics, path: str = DEFAULT_PATH) -> str:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, **{f.name: getattr(go, f.name) for f in fields(go)})
    return path


def load(path: str = DEFAULT_PATH) -> GasOptics:
    with np.load(path) as z:
        return GasOptics(**{f.name: z[f.name] for f in fields(GasOptics)}).validate()


def load_default() -> GasOptics | None:
    """The tables saved at :data:`DEFAULT_PATH` (written by the package build
    from a reference checkout), or None."""
    return load(DEFAULT_PATH) if os.path.exists(DEFAULT_PATH) else None


# ---- synthetic tables -----------------------------------------------------------------------

def _band_planck(t: np.ndarray, nu_lo: float, nu_hi: float, n: int = 64) -> np.ndarray:
    """Planck radiance integrated over wavenumbers [nu_lo, nu_hi] (1/m),
    W/m2/sr, by the midpoint rule."""
    h, c, k = 6.62607015e-34, 2.99792458e8, 1.380649e-23
    nu = nu_lo + (np.arange(n) + .5) * (nu_hi - nu_lo) / n
    x = h * c * nu[None, :] / (k * t[:, None])
    b = 2 * h * c ** 2 * nu[None, :] ** 3 / np.expm1(x)
    return b.sum(axis=1) * (nu_hi - nu_lo) / n


def synthetic(seed: int = 0, n_g: int = 16, n_p: int = 53, n_t: int = 6, n_planck: int = 231) -> GasOptics:
    """Tables with the reference's shapes and plausible magnitudes: pressures
    log-spaced from 1 Pa to 1.1e5 Pa, a temperature grid of n_t points 20 K
    apart centred on a standard-atmosphere profile, absorption coefficients
    rising with pressure and temperature over several decades across the
    g-points, Planck functions of 16 longwave bands on 120-350 K."""
    rng = np.random.default_rng(seed)
    p = np.geomspace(1.0, 1.1e5, n_p)
    zkm = -7.0 * np.log(p / 1.0e5)
    tref = np.where(zkm < 11, 288.0 - 6.5 * zkm, 216.65) + 8.0 * np.clip(zkm - 20, 0, 30) / 30
    temps = tref[:, None] + 20.0 * (np.arange(n_t) - (n_t - 1) / 2)[None, :]
    scale_sw = 10.0 ** np.linspace(-6, 0, n_g) * rng.uniform(.5, 2, n_g)
    scale_lw = 10.0 ** np.linspace(-4, 1.5, n_g) * rng.uniform(.5, 2, n_g)
    shape_p = (p / 1.0e5)[None, :, None] ** rng.uniform(.3, 1.0, (n_g, 1, 1))
    shape_t = (temps / 250.0)[None, :, :] ** rng.uniform(-1, 2, (n_g, 1, 1))
    sw = scale_sw[:, None, None] * (.05 + shape_p) * shape_t
    lw = scale_lw[:, None, None] * (.05 + shape_p) * shape_t
    sca = 10.0 ** np.linspace(-7, -4, n_g) * rng.uniform(.5, 2, n_g)
    pt = np.linspace(120.0, 350.0, n_planck)
    edges = np.linspace(1.0e3, 3.0e5, n_g + 1)  # 10-3000 cm-1
    planck = np.stack([_band_planck(pt, edges[g], edges[g + 1]) for g in range(n_g)])
    frac = rng.uniform(.2, 1.0, n_g)
    frac = frac / frac.sum()
    return GasOptics(p, temps, sw, sca, lw, pt, planck, frac).validate()
