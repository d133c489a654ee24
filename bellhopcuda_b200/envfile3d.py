"""Writers for BELLHOP3D input files: the 3-D .env, the hexahedral .ssp and the
'R' (rectangular grid) altimetry / bathymetry files.

Formats follow the reference's readers: the 3-D .env adds source x / y
(src/module/sxsy.hpp), receiver bearings (src/module/rcvrbearings.hpp), the
bearing fan (src/module/rayangles.hpp) and a three-dimensional beam box
(src/module/beaminfo.hpp) to the 2-D layout; the hexahedral .ssp holds Nx, x
(km), Ny, y (km), Nz, z (m) and one record of Nx sound speeds per (z, y)
(src/module/ssp.hpp:144-186); a grid boundary holds its type, Nx, x (km), Ny,
y (km) and one row of Nx depths per y (src/module/boundary.hpp:105-147).
"""
from __future__ import annotations

import os
from typing import Dict, Optional, Sequence, Tuple

import numpy as np


def _vec(vals) -> str:
    return " ".join("%.6f" % v for v in vals) + " /"


def env_text(*, title: str, freq: float, ssp_opt: str, depth: float, ssp: Sequence[Tuple[float, float]],
             bot: tuple, sx: Sequence[float], sy: Sequence[float], sz: Sequence[float],
             rz: Optional[Sequence[float]], rr_km: Optional[Sequence[float]], theta: Sequence[float],
             run_type: str, alpha: tuple, beta: tuple, step: float, box_km: Tuple[float, float], box_z: float,
             nrz_range: Optional[tuple] = None, rr_range: Optional[tuple] = None,
             theta_range: Optional[tuple] = None) -> str:
    """One BELLHOP3D .env. ``bot`` is (option,) or ("A", cp, rho, atten) for a
    halfspace; receivers / bearings are explicit lists or (n, first, last)
    ranges that the reader fills in (SubTab). Options are written verbatim:
    a '~' in ``bot[0]`` or the fifth character of ``ssp_opt`` asks for a
    bathymetry / altimetry file."""
    L = ["'%s'" % title, "%g" % freq, "1", "'%s'" % ssp_opt, "0 0.0 %g" % depth]
    L += ["%g %g /" % (z, c) for z, c in ssp]
    L += ["'%s' 0.0" % bot[0]]
    if bot[0][0] == "A":
        L += ["%g %g 0.0 %g %g /" % (depth, bot[1], bot[2], bot[3])]
    L += ["%d" % len(sx), _vec(sx), "%d" % len(sy), _vec(sy), "%d" % len(sz), _vec(sz)]
    L += ["%d" % nrz_range[0], "%g %g /" % tuple(nrz_range[1:])] if nrz_range else ["%d" % len(rz), _vec(rz)]
    L += ["%d" % rr_range[0], "%g %g /" % tuple(rr_range[1:])] if rr_range else ["%d" % len(rr_km), _vec(rr_km)]
    if theta_range:
        L += ["%d" % theta_range[0], "%g %g /" % tuple(theta_range[1:])]
    else:
        L += ["%d" % len(theta), _vec(theta)]
    L += ["'%s'" % run_type]
    L += ["%d" % alpha[0], "%g %g /" % tuple(alpha[1:])]
    L += ["%d" % beta[0], "%g %g /" % tuple(beta[1:])]
    L += ["%g %g %g %g" % (step, box_km[0], box_km[1], box_z)]
    return "\n".join(L) + "\n"


def grid_text(x_km, y_km, z, kind="R") -> str:
    """Altimetry / bathymetry grid ('R' flat triangles, 'C' curvilinear):
    z[ix, iy] in m, one row per y."""
    L = ["'%s'" % kind, "%d" % len(x_km), _vec(x_km), "%d" % len(y_km), _vec(y_km)]
    for iy in range(len(y_km)):
        L.append(" ".join("%.4f" % z[ix, iy] for ix in range(len(x_km))))
    return "\n".join(L) + "\n"


def hex_ssp_text(x_km, y_km, z, c) -> str:
    """Hexahedral .ssp: c[ix, iy, iz] in m/s, one record per (iz, iy) of Nx values."""
    L = ["%d" % len(x_km), " ".join("%.6f" % v for v in x_km), "%d" % len(y_km),
         " ".join("%.6f" % v for v in y_km), "%d" % len(z), " ".join("%.6f" % v for v in z)]
    for iz in range(len(z)):
        for iy in range(len(y_km)):
            L.append(" ".join("%.4f" % c[ix, iy, iz] for ix in range(len(x_km))))
    return "\n".join(L) + "\n"


def write_files(files: Dict[str, str], root: str) -> str:
    """Write {suffix: text} next to ``root``; returns root."""
    d = os.path.dirname(root)
    if d:
        os.makedirs(d, exist_ok=True)
    for suffix, text in files.items():
        with open(root + suffix, "w") as f:
            f.write(text)
    return root
