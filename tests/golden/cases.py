"""Small deterministic environments used for the golden fixtures and the
oracle / GPU parity tests. Each case is a function returning an EnvSpec."""
from __future__ import annotations

import numpy as np

from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import EnvSpec


def _small(spec, nrz=31, nrr=101, nalpha=151):
    spec.nrz, spec.nrr, spec.nalpha = nrz, nrr, nalpha
    return spec


def munk_hat():
    return _small(W.munk_tl())


def munk_gauss():
    return _small(W.munk_tl(beam="B"))


def munk_incoherent():
    s = _small(W.munk_tl())
    s.run_type = "IG RR "
    return s


def munk_semicoherent_gauss():
    s = _small(W.munk_tl(beam="B"))
    s.run_type = "SB RR "
    return s


def munk_n2linear():
    s = _small(W.munk_tl())
    s.ssp_type = "N"
    return s


def munk_spline_rigid():
    s = _small(W.munk_tl(beam="B"))
    s.ssp_type = "S"
    s.bot_bc = "R"
    return s


def rd_pchip_bty():
    return _small(W.rd_gauss(nalpha=151, nrz=31, nrr=101, nbty=40))


def rd_curvilinear_ati():
    rng = np.random.Generator(np.random.PCG64(7))
    s = _small(W.rd_gauss(nalpha=151, nrz=31, nrr=101, nbty=30))
    s.bty_type = "CS"
    s.ati_r = list(np.linspace(0.0, 100.0, 25))
    s.ati_z = list(rng.uniform(0.0, 30.0, 25))
    s.ati_type = "LS"
    s.sz = (500.0,)
    return s


def shallow_long_bty_grain():
    """Shallow water, long-format bathymetry (per-segment halfspace) and a
    grain-size top is not physical; use an elastic 'A' bottom with shear."""
    rng = np.random.Generator(np.random.PCG64(11))
    z = np.linspace(0.0, 200.0, 21)
    c = 1510.0 - 0.05 * z + rng.normal(0.0, 0.5, z.size)
    br = list(np.linspace(0.0, 10.0, 12))
    bz = list(rng.uniform(150.0, 200.0, 12))
    geo = [[float(rng.uniform(1550, 1750)), 0.0, float(rng.uniform(1.4, 2.0)), 0.5, 0.0] for _ in br]
    return EnvSpec(title="shallow long bty", freq=250.0, ssp_type="C", top_bc="V", atten_unit="W",
                   ssp_z=z, ssp_cp=c, bot_bc="A", bot_hs=(200.0, 1700.0, 400.0, 1.9, 0.5, 0.2),
                   bty_r=br, bty_z=bz, bty_type="LL", bty_geo=geo, nsz=2, sz=(20.0, 80.0),
                   nrz=21, rz=(0.0, 200.0), nrr=81, rr_km=(0.0, 10.0), run_type="CB RR ",
                   nalpha=201, alpha=(-40.0, 40.0), deltas=0.0, box_z=250.0, box_r_km=10.5)


def thorp_line_source():
    s = _small(W.munk_tl())
    s.vol_atten = "T"
    s.run_type = "CG XR "
    return s


CASES = {f.__name__: f for f in [munk_hat, munk_gauss, munk_incoherent, munk_semicoherent_gauss,
                                  munk_n2linear, munk_spline_rigid, rd_pchip_bty, rd_curvilinear_ati,
                                  shallow_long_bty_grain, thorp_line_source]}
