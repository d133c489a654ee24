"""2-D golden cases for the options beyond the oracle restatement (quad SSP,
reflection-coefficient tables, beam shift, further beam types): small
environments written as the reference's input files.

Each case is a dict of file suffix -> text (.env plus the side files the
option reads: .ssp for the quad SSP, .brc / .trc for tabulated reflection
coefficients, .bty / .ati). The fixtures of these cases are made by running
the reference's own bellhopcxx on them (tests/golden/make_golden_ext.py).
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from bellhopcuda_b200.envfile import EnvSpec, _bdry_text, env_text  # noqa: E402
from bellhopcuda_b200.workloads import munk_c  # noqa: E402


def quad_ssp_text(r_km, c):
    """The quad SSP file: Nr, the profile ranges (km), then one row of Nr
    sound speeds per depth of the .env profile (src/module/ssp.hpp:122-141)."""
    c = np.asarray(c, dtype=np.float64)
    lines = [str(len(r_km)), " ".join(repr(float(v)) for v in r_km)]
    for row in c:
        lines.append(" ".join(repr(float(v)) for v in row))
    return "\n".join(lines) + "\n"


def _quad_munk(run_type, nalpha=301, **kw):
    """Munk channel whose axis deepens from 1000 m to 1600 m over 60 km,
    sampled as 5 range profiles on the .env depths."""
    z = np.arange(0.0, 5000.0 + 1e-9, 250.0)
    r_km = np.array([-1.0, 15.0, 30.0, 45.0, 61.0])
    c = np.stack([munk_c(z - 10.0 * max(r, 0.0)) for r in r_km], axis=1)
    spec = EnvSpec(title="quad Munk", freq=50.0, ssp_type="Q", top_bc="V", atten_unit="W",
                   ssp_z=z, ssp_cp=c[:, 0], bot_bc="A", bot_hs=(5000.0, 1600.0, 0.0, 1.8, 0.8, 0.0),
                   nsz=1, sz=(1000.0,), nrz=51, rz=(0.0, 5000.0), nrr=201, rr_km=(0.0, 60.0),
                   run_type=run_type, nalpha=nalpha, alpha=(-20.0, 20.0), deltas=0.0, box_z=5500.0,
                   box_r_km=60.5)
    for k, v in kw.items():
        setattr(spec, k, v)
    return {".env": env_text(spec), ".ssp": quad_ssp_text(r_km, c)}


def quad_munk_gauss():
    return _quad_munk("CB RR ")


def quad_munk_hat():
    return _quad_munk("CG RR ")


def quad_munk_incoherent():
    return _quad_munk("IG RR ")


def quad_shallow_bty():
    """Shallow water with a warm front: the sound speed drops 25 m/s over
    10 km in the upper 60 m, over a sloping bathymetry; hat beams, two sources."""
    z = np.array([0.0, 20.0, 40.0, 60.0, 80.0, 120.0, 200.0])
    r_km = np.array([0.0, 4.0, 8.0, 12.0, 16.0, 20.5])
    base = np.array([1530.0, 1528.0, 1520.0, 1505.0, 1495.0, 1492.0, 1490.0])
    drop = np.array([25.0, 24.0, 18.0, 8.0, 2.0, 0.0, 0.0])
    frac = np.clip(r_km / 10.0, 0.0, 1.0)
    c = base[:, None] - drop[:, None] * frac[None, :]
    spec = EnvSpec(title="quad front", freq=250.0, ssp_type="Q", top_bc="V", atten_unit="W",
                   ssp_z=z, ssp_cp=c[:, 0], bot_bc="A", bot_hs=(200.0, 1650.0, 0.0, 1.7, 0.6, 0.0),
                   nsz=2, sz=(25.0, 90.0), nrz=41, rz=(0.0, 200.0), nrr=161, rr_km=(0.0, 20.0),
                   run_type="CG RR ", nalpha=401, alpha=(-45.0, 45.0), deltas=0.0, box_z=210.0,
                   box_r_km=20.2)
    bty_r = np.array([-1.0, 5.0, 12.0, 21.0])
    bty_z = np.array([180.0, 160.0, 130.0, 150.0])
    spec.bty_r, spec.bty_z = bty_r, bty_z
    return {".env": env_text(spec), ".ssp": quad_ssp_text(r_km, c), ".bty": _bdry_text("LS", bty_r, bty_z, None)}


def rayleigh_table(c1, c2, rho2, att_db_wl, thetas_deg):
    """|R| and phase (deg) of a fluid halfspace under water (density 1) against
    the grazing angle, written as a .brc / .trc table: NPts, then
    (theta, |R|, phase) triples (src/module/reflcoef.hpp:50-75)."""
    th = np.deg2rad(np.asarray(thetas_deg, dtype=np.float64))
    c2c = c2 / (1.0 + 1j * att_db_wl / (40.0 * np.pi * np.log10(np.e)))
    kz1 = np.sin(th) / c1
    kz2 = np.sqrt((1.0 / c2c) ** 2 - (np.cos(th) / c1) ** 2 + 0j)
    R = (rho2 * kz1 - kz2) / (rho2 * kz1 + kz2)
    phase = np.degrees(np.unwrap(np.angle(R)))
    lines = [str(len(th))]
    for t, r, ph in zip(thetas_deg, R, phase):
        lines.append("%r %r %r" % (float(t), float(abs(r)), float(ph)))
    return "\n".join(lines) + "\n"


def _munk_spec(**kw):
    z = np.arange(0.0, 5000.0 + 1e-9, 100.0)
    spec = EnvSpec(title="Munk table bottom", freq=50.0, ssp_type="C", top_bc="V", atten_unit="W",
                   ssp_z=z, ssp_cp=munk_c(z), bot_bc="F", nsz=1, sz=(1000.0,), nrz=51, rz=(0.0, 5000.0),
                   nrr=201, rr_km=(0.0, 50.0), run_type="CB RR ", nalpha=401, alpha=(-45.0, 45.0),
                   deltas=0.0, box_z=5500.0, box_r_km=51.0)
    for k, v in kw.items():
        setattr(spec, k, v)
    return spec


def brc_munk_gauss():
    """Munk channel over a tabulated bottom (fluid halfspace 1600 m/s, 1.8
    g/cm3, 0.8 dB/wavelength, tabulated every 2 degrees)."""
    spec = _munk_spec()
    return {".env": env_text(spec), ".brc": rayleigh_table(1551.91, 1600.0, 1.8, 0.8, np.arange(0.0, 90.1, 2.0))}


def trc_brc_shallow_hat():
    """Shallow water with both boundaries tabulated: a lossy surface (|R| from
    0.99 at grazing to 0.9 at normal incidence, phase 180 deg) and a sand
    bottom; hat beams, two sources."""
    z = np.array([0.0, 30.0, 60.0, 100.0])
    c = np.array([1520.0, 1515.0, 1495.0, 1490.0])
    spec = EnvSpec(title="tabulated shallow", freq=200.0, ssp_type="C", top_bc="F", atten_unit="W",
                   ssp_z=z, ssp_cp=c, bot_bc="F", nsz=2, sz=(20.0, 70.0), nrz=41, rz=(0.0, 100.0), nrr=161,
                   rr_km=(0.0, 8.0), run_type="CG RR ", nalpha=301, alpha=(-60.0, 60.0), deltas=0.0,
                   box_z=110.0, box_r_km=8.1)
    th = np.arange(0.0, 90.1, 5.0)
    trc = [str(len(th))] + ["%r %r 180.0" % (float(t), float(0.99 - 0.09 * t / 90.0)) for t in th]
    return {".env": env_text(spec), ".trc": "\n".join(trc) + "\n",
            ".brc": rayleigh_table(1490.0, 1700.0, 1.9, 0.5, np.arange(0.0, 90.1, 1.0))}


def trc_brc_shallow_incoherent():
    f = trc_brc_shallow_hat()
    f[".env"] = f[".env"].replace("'CG RR'", "'IG RR'")
    return f


def beam_shift_shallow():
    """Beam displacement on halfspace reflections (RunType(7) = 'S'), shallow
    water over a sloping sand bottom, Gaussian beams."""
    z = np.array([0.0, 30.0, 60.0, 120.0])
    c = np.array([1520.0, 1515.0, 1495.0, 1490.0])
    spec = EnvSpec(title="beam shift shallow", freq=300.0, ssp_type="C", top_bc="V", atten_unit="W",
                   ssp_z=z, ssp_cp=c, bot_bc="A", bot_hs=(120.0, 1700.0, 0.0, 1.9, 0.5, 0.0), nsz=1,
                   sz=(40.0,), nrz=41, rz=(0.0, 120.0), nrr=161, rr_km=(0.0, 8.0), run_type="CB RR S",
                   nalpha=301, alpha=(-50.0, 50.0), deltas=0.0, box_z=130.0, box_r_km=8.1)
    spec.bty_r, spec.bty_z = np.array([-1.0, 3.0, 9.0]), np.array([100.0, 80.0, 110.0])
    return {".env": env_text(spec), ".bty": _bdry_text("LS", spec.bty_r, spec.bty_z, None)}


def beam_shift_munk_hat():
    spec = _munk_spec(bot_bc="A", bot_hs=(5000.0, 1600.0, 0.0, 1.8, 0.8, 0.0), run_type="CG RR S")
    return {".env": env_text(spec)}


def _with_beam_lines(files, width_curv="MS", eps_mult=1.0, rloop=10.0, nimage=1, ibwin=5, comp="P"):
    """Append the Cerveny beam records (src/module/beaminfo.hpp:79-90): width /
    curvature options, epsilon multiplier, rLoop (km), then the number of
    images, beam window and field component."""
    files[".env"] = files[".env"] + "'%s' %r %r\n%d %d '%s'\n" % (width_curv, float(eps_mult), float(rloop), nimage,
                                                                 ibwin, comp)
    return files


def _munk_small(run_type, **kw):
    spec = _munk_spec(bot_bc="A", bot_hs=(5000.0, 1600.0, 0.0, 1.8, 0.8, 0.0), run_type=run_type, nalpha=301,
                      alpha=(-20.0, 20.0), rr_km=(0.0, 50.0), nrr=201, nrz=51)
    for k, v in kw.items():
        setattr(spec, k, v)
    return {".env": env_text(spec)}


def _shallow_small(run_type, **kw):
    z = np.array([0.0, 30.0, 60.0, 100.0])
    c = np.array([1520.0, 1515.0, 1495.0, 1490.0])
    spec = EnvSpec(title="shallow beams", freq=200.0, ssp_type="C", top_bc="V", atten_unit="W", ssp_z=z,
                   ssp_cp=c, bot_bc="A", bot_hs=(100.0, 1700.0, 0.0, 1.9, 0.5, 0.0), nsz=2, sz=(20.0, 70.0), nrz=41,
                   rz=(0.0, 100.0), nrr=161, rr_km=(0.0, 8.0), run_type=run_type, nalpha=301, alpha=(-60.0, 60.0),
                   deltas=0.0, box_z=110.0, box_r_km=8.1)
    for k, v in kw.items():
        setattr(spec, k, v)
    return {".env": env_text(spec)}


CASES2D_EXT = {
    "x2d_quad_munk_gauss": quad_munk_gauss,
    "x2d_quad_munk_hat": quad_munk_hat,
    "x2d_quad_munk_incoherent": quad_munk_incoherent,
    "x2d_quad_shallow_bty": quad_shallow_bty,
    "x2d_brc_munk_gauss": brc_munk_gauss,
    "x2d_trc_brc_shallow_hat": trc_brc_shallow_hat,
    "x2d_trc_brc_shallow_incoherent": trc_brc_shallow_incoherent,
    "x2d_beam_shift_shallow": beam_shift_shallow,
    "x2d_beam_shift_munk_hat": beam_shift_munk_hat,
    # geometric beams in ray-centred coordinates ('g' hat, 'b' Gaussian)
    "x2d_raycen_hat_munk": lambda: _munk_small("Cg RR "),
    "x2d_raycen_gauss_munk": lambda: _munk_small("Cb RR "),
    "x2d_raycen_hat_shallow_incoherent": lambda: _shallow_small("Ig RR "),
    "x2d_raycen_gauss_shallow_semicoherent": lambda: _shallow_small("Sb RR "),
    # Cerveny paraxial beams: ray-centred ('R') and Cartesian ('C')
    "x2d_cerveny_raycen_munk": lambda: _with_beam_lines(_munk_small("CR RR ")),
    "x2d_cerveny_cart_munk": lambda: _with_beam_lines(_munk_small("CC RR ")),
    "x2d_cerveny_raycen_shallow_images": lambda: _with_beam_lines(_shallow_small("CR RR "), "FS", 1.0, 1.0, 3, 4),
    "x2d_cerveny_cart_shallow_images_incoherent": lambda: _with_beam_lines(_shallow_small("IC RR "), "FD", 0.5, 1.0,
                                                                           2, 4),
    "x2d_cerveny_raycen_wkb_vertical": lambda: _with_beam_lines(_munk_small("CR RR "), "WS", 1.0, 10.0, 1, 5, "V"),
    # simple Gaussian beams ('S')
    "x2d_sgb_munk": lambda: _munk_small("CS RR "),
    "x2d_sgb_shallow_incoherent": lambda: _shallow_small("IS RR "),
    # arrivals (binary .arr) and eigen hits (the .ray of the re-traced hit rays)
    # with ray-centred geometric and simple Gaussian beams
    "x2d_arr_raycen_hat_munk": lambda: _munk_small("ag RR ", nrz=11, nrr=21),
    "x2d_arr_raycen_gauss_shallow": lambda: _shallow_small("ab RR ", nrz=6, nrr=11, nalpha=151),
    "x2d_arr_sgb_munk": lambda: _munk_small("aS RR ", nrz=6, nrr=11),
    "x2d_arr_sgb_shallow": lambda: _shallow_small("aS RR ", nrz=6, nrr=11, nalpha=151),
    "x2d_eig_raycen_hat_munk": lambda: _munk_small("Eg RR ", nrz=3, rz=(800.0, 3000.0), nrr=4, rr_km=(20.0, 50.0)),
    "x2d_eig_raycen_gauss_shallow": lambda: _shallow_small("Eb RR ", nrz=3, rz=(25.0, 75.0), nrr=3,
                                                           rr_km=(3.0, 7.0)),
    "x2d_eig_sgb_munk": lambda: _munk_small("ES RR ", nrz=3, rz=(800.0, 3000.0), nrr=4, rr_km=(20.0, 50.0)),
    # arrivals and eigen hits in one run ('v': binary .arr and the .ray of the hits)
    "x2d_arr_v_cart_hat_munk": lambda: _munk_small("vG RR ", nrz=3, rz=(800.0, 3000.0), nrr=4, rr_km=(20.0, 50.0)),
    "x2d_arr_v_raycen_gauss_shallow": lambda: _shallow_small("vb RR ", nrz=3, rz=(25.0, 75.0), nrr=3,
                                                             rr_km=(3.0, 7.0)),
}
