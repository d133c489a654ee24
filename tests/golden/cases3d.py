"""3-D (BELLHOP3D) golden cases: small environments written as the reference's
input files (.env, plus .ssp for the hexahedral grid and .bty / .ati grids).

Each case is a dict of file suffix -> text. The shapes follow the reference's
own 3-D test environments (Munk slice, hexahedral Munk, seamount and
paraboloid grids), scaled down so that the reference traces each in seconds.
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from bellhopcuda_b200.envfile3d import env_text, grid_text, hex_ssp_text  # noqa: E402

MUNK = [(0.0, 1548.52), (200.0, 1530.29), (250.0, 1526.69), (400.0, 1517.78), (600.0, 1509.49),
        (800.0, 1504.30), (1000.0, 1501.38), (1200.0, 1500.14), (1400.0, 1500.12), (1600.0, 1501.02),
        (1800.0, 1502.57), (2000.0, 1504.62), (2200.0, 1507.02), (2400.0, 1509.69), (2600.0, 1512.55),
        (2800.0, 1515.56), (3000.0, 1518.67), (3200.0, 1521.85), (3400.0, 1525.10), (3600.0, 1528.38),
        (3800.0, 1531.70), (4000.0, 1535.04), (4200.0, 1538.39), (4400.0, 1541.76), (4600.0, 1545.14),
        (4800.0, 1548.52), (5000.0, 1551.91)]


def _munk_slice(run_type, **kw):
    args = dict(title="Munk slice 3-D", freq=50.0, ssp_opt="CVW", depth=5000.0, ssp=MUNK,
                bot=("A", 1600.0, 1.8, 0.8), sx=[0.0], sy=[0.0], sz=[1000.0], rz=None, rr_km=None,
                theta=[0.0, 2.0, 5.0], run_type=run_type, alpha=(121, -20.3, 20.3), beta=(21, -8.0, 8.0),
                step=200.0, box_km=(31.0, 31.0), box_z=5500.0, nrz_range=(51, 0.0, 5000.0),
                rr_range=(101, 0.0, 30.0))
    args.update(kw)
    return {".env": env_text(**args)}


def munk3d_gauss():
    return _munk_slice("CB   3")


def munk3d_hat():
    return _munk_slice("CG   3")


def munk3d_hat_incoherent():
    return _munk_slice("IG   3")


def munk3d_gauss_semicoherent():
    return _munk_slice("SB   3")


def munk3d_sources():
    """Several sources in x, y and z: exercises the job and field layouts."""
    return _munk_slice("CB   3", sx=[0.0, 1.0], sy=[-0.5, 0.5], sz=[800.0, 1500.0], alpha=(61, -15.0, 15.0),
                       beta=(11, -6.0, 6.0), theta=[0.0, 3.0], rr_range=(61, 0.0, 20.0), box_km=(25.0, 25.0))


def hex3d_gauss():
    """Hexahedral SSP: a Munk profile whose axis deepens along x and tilts in y."""
    xs = np.array([-30.0, 0.0, 30.0])
    ys = np.array([-30.0, 0.0, 30.0])
    z = np.array([0.0, 500.0, 1000.0, 1500.0, 2500.0, 3500.0, 5000.0])
    zp, cp = np.array(MUNK).T
    c = np.zeros((3, 3, len(z)))
    for ix, x in enumerate(xs):
        for iy, y in enumerate(ys):
            shift = 8.0 * x + 4.0 * y          # m of axis depth per km
            c[ix, iy] = np.interp(z - shift, zp, cp)
    env = env_text(title="hexahedral Munk", freq=50.0, ssp_opt="HVW", depth=5000.0,
                   ssp=[(float(zz), 1500.0) for zz in z], bot=("A", 1600.0, 1.8, 0.8), sx=[0.0], sy=[0.0],
                   sz=[1000.0], rz=None, rr_km=None, theta=[0.0, 3.0, 90.0], run_type="CB   3",
                   alpha=(101, -18.0, 18.0), beta=(31, -12.0, 12.0), step=200.0, box_km=(25.0, 25.0),
                   box_z=5500.0, nrz_range=(41, 0.0, 5000.0), rr_range=(81, 0.0, 20.0))
    return {".env": env, ".ssp": hex_ssp_text(xs, ys, z, c)}


def seamount3d_gauss():
    """Gaussian seamount on an 'R' bathymetry grid, halfspace bottom."""
    xs = np.linspace(-12.0, 12.0, 25)
    ys = np.linspace(-12.0, 12.0, 25)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    z = 3000.0 - 2200.0 * np.exp(-((X - 5.0) ** 2 + (Y - 1.0) ** 2) / 4.0)
    env = env_text(title="seamount 3-D", freq=100.0, ssp_opt="CVW", depth=3000.0,
                   ssp=[(0.0, 1500.0), (3000.0, 1500.0)], bot=("A", 1650.0, 1.5, 0.5), sx=[0.0], sy=[0.0],
                   sz=[250.0], rz=[400.0, 1000.0], rr_km=None, theta=[0.0, 10.0, 20.0, 350.0], run_type="CB   3",
                   alpha=(91, -30.0, 30.0), beta=(73, -180.0, 180.0), step=100.0, box_km=(11.0, 11.0),
                   box_z=3100.0, rr_range=(101, 0.0, 10.0))
    return {".env": env.replace("'A' 0.0", "'A~' 0.0"), ".bty": grid_text(xs, ys, z)}


def parabot3d_hat():
    """Paraboloid altimetry-free bottom grid with hat beams and a rigid-free mix."""
    xs = np.linspace(-6.0, 6.0, 13)
    ys = np.linspace(-6.0, 6.0, 13)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    z = 600.0 + 12.0 * (X ** 2 + Y ** 2)
    env = env_text(title="paraboloid bowl", freq=200.0, ssp_opt="CVW", depth=1100.0,
                   ssp=[(0.0, 1500.0), (1100.0, 1500.0)], bot=("R",), sx=[0.0], sy=[0.0], sz=[100.0],
                   rz=None, rr_km=None, theta=[0.0, 45.0, 90.0], run_type="CG   3", alpha=(61, -40.0, 40.0),
                   beta=(37, 0.0, 360.0), step=50.0, box_km=(5.5, 5.5), box_z=1200.0, nrz_range=(21, 0.0, 1000.0),
                   rr_range=(51, 0.0, 5.0))
    return {".env": env.replace("'R' 0.0", "'R~' 0.0"), ".bty": grid_text(xs, ys, z)}


def munk3d_arr_gauss():
    """Arrivals ('a', binary) on a sparse receiver grid."""
    return _munk_slice("aB   3", alpha=(121, -20.3, 20.3), beta=(21, -8.0, 8.0), theta=[0.0, 2.0, 5.0],
                       nrz_range=(6, 500.0, 3000.0), rr_range=(7, 5.0, 30.0))


def munk3d_arr_hat():
    return _munk_slice("aG   3", alpha=(121, -20.3, 20.3), beta=(21, -8.0, 8.0), theta=[0.0, 3.0],
                       nrz_range=(5, 800.0, 2800.0), rr_range=(6, 8.0, 28.0))


def parabot3d_arr_hat():
    """Arrivals with many bottom bounces off a gridded bowl."""
    f = parabot3d_hat()
    f[".env"] = f[".env"].replace("'CG   3'", "'aG   3'").replace("21\n0 1000 /", "4\n200 800 /").replace(
        "51\n0 5 /", "6\n1 5 /")
    return f


def munk3d_eig_gauss():
    """Eigenray hits ('E') on a sparse receiver grid."""
    return _munk_slice("EB   3", alpha=(121, -20.3, 20.3), beta=(21, -8.0, 8.0), theta=[0.0, 2.0, 5.0],
                       nrz_range=(3, 800.0, 2800.0), rr_range=(4, 8.0, 26.0))


def seamount3d_eig_hat():
    f = seamount3d_gauss()
    f[".env"] = f[".env"].replace("'CB   3'", "'EG   3'").replace("101\n0 10 /", "3\n3 9 /")
    return f


def munk3d_brc_gauss():
    """Munk slice over a tabulated bottom reflection coefficient (.brc)."""
    from cases2d_ext import rayleigh_table
    f = _munk_slice("CB   3", bot=("F",))
    f[".brc"] = rayleigh_table(1551.91, 1600.0, 1.8, 0.8, np.arange(0.0, 90.1, 2.0))
    return f


def munk3d_ray():
    """Ray trajectories ('R'), 3-D: a small fan in elevation and bearing."""
    return _munk_slice("R    3", alpha=(11, -12.0, 12.0), beta=(5, -6.0, 6.0), theta=[0.0])


def seamount3d_ray():
    """Ray trajectories over the seamount grid (bottom reflections off the
    triangulated bathymetry)."""
    f = seamount3d_gauss()
    f[".env"] = f[".env"].replace("'CB   3'", "'R    3'").replace("91\n-30 30 /", "9\n-30 30 /").replace(
        "73\n-180 180 /", "12\n-180 180 /")
    return f


def munk3d_raycen_hat():
    """Geometric hat beams in ray-centred coordinates ('g')."""
    return _munk_slice("Cg   3")


def munk3d_raycen_gauss():
    """Geometric Gaussian beams in ray-centred coordinates ('b')."""
    return _munk_slice("Cb   3")


def seamount3d_raycen_hat():
    f = seamount3d_gauss()
    f[".env"] = f[".env"].replace("'CB   3'", "'Cg   3'")
    return f


def parabot3d_raycen_incoherent():
    f = parabot3d_hat()
    f[".env"] = f[".env"].replace("'CG   3'", "'Ig   3'")
    return f


def munk3d_nx2d_gauss():
    """Nx2D (RunType(6) '2'): 2-D Gaussian beams along each receiver bearing of
    the Munk slice."""
    return _munk_slice("CB   2")


def hex3d_nx2d_hat():
    """Nx2D through the hexahedral SSP (range- and bearing-dependent channel)."""
    f = hex3d_gauss()
    f[".env"] = f[".env"].replace("'CB   3'", "'CG   2'")
    return f


def seamount3d_nx2d_gauss():
    """Nx2D over the seamount grid: bottom reflections off the triangles
    projected on each bearing's plane."""
    f = seamount3d_gauss()
    f[".env"] = f[".env"].replace("'CB   3'", "'CB   2'")
    return f


def parabot3d_nx2d_incoherent():
    f = parabot3d_hat()
    f[".env"] = f[".env"].replace("'CG   3'", "'IG   2'")
    return f


def _curvilinear(files):
    """The same boundary grid read as curvilinear ('C'): reflections use the
    normal interpolated between the node normals and the cell's curvature."""
    files[".bty"] = files[".bty"].replace("'R'", "'C'", 1)
    return files


def parabot3d_curv_hat():
    return _curvilinear(parabot3d_hat())


def seamount3d_curv_gauss():
    return _curvilinear(seamount3d_gauss())


def parabot3d_curv_nx2d():
    return _curvilinear(parabot3d_nx2d_incoherent())


def munk3d_nx2d_ray():
    """Nx2D ray run: 2-D rays in the planes of the bearing fan (not replaced by
    the receiver bearings for ray runs), points written in (x, y, z)."""
    return _munk_slice("R    2", alpha=(11, -12.0, 12.0), beta=(5, -6.0, 6.0), theta=[0.0])


def munk3d_nx2d_arr_gauss():
    """Nx2D arrivals ('a', binary): the 2-D Gaussian beams of each receiver
    bearing's plane as arrivals, cylindrical spreading per range."""
    return _munk_slice("aB   2", alpha=(121, -20.3, 20.3), theta=[0.0, 2.0, 5.0], nrz_range=(6, 500.0, 3000.0),
                       rr_range=(7, 5.0, 30.0))


def munk3d_raycen_arr_gauss():
    """Arrivals ('a') of Gaussian beams in ray-centred coordinates ('b'),
    the depth / bearing / range walk of Step_InfluenceGeoRayCen."""
    return _munk_slice("ab   3", nrz_range=(6, 500.0, 3000.0), rr_range=(7, 5.0, 30.0))


def munk3d_raycen_eig_hat():
    """Eigen hits ('E') of hat beams in ray-centred coordinates ('g')."""
    return _munk_slice("Eg   3", alpha=(121, -20.3, 20.3), beta=(21, -8.0, 8.0), theta=[0.0, 2.0, 5.0],
                       nrz_range=(3, 800.0, 2800.0), rr_range=(4, 8.0, 26.0))


def munk3d_nx2d_eig_gauss():
    """Nx2D eigen hits ('E'): the hits of each receiver bearing's plane
    (itheta = ibeta), on a sparse receiver grid."""
    return _munk_slice("EB   2", alpha=(121, -20.3, 20.3), theta=[0.0, 2.0, 5.0], nrz_range=(3, 800.0, 2800.0),
                       rr_range=(4, 8.0, 26.0))


def seamount3d_nx2d_arr_hat():
    """Nx2D arrivals with hat beams over the seamount grid on four bearings
    (reflections off the triangles projected on each plane)."""
    f = seamount3d_gauss()
    f[".env"] = f[".env"].replace("'CB   3'", "'aG   2'").replace("101\n0 10 /", "11\n0 10 /")
    return f


def seamount3d_nx2d_ray():
    f = seamount3d_ray()
    f[".env"] = f[".env"].replace("'R    3'", "'R    2'")
    return f


def munk3d_v_hat():
    """Arrivals and eigen hits in one run ('v', binary arrivals) with hat beams."""
    return _munk_slice("vG   3", alpha=(121, -20.3, 20.3), beta=(21, -8.0, 8.0), theta=[0.0, 2.0, 5.0],
                       nrz_range=(3, 800.0, 2800.0), rr_range=(4, 8.0, 26.0))


def munk3d_raycen_v_gauss():
    """'v' with Gaussian beams in ray-centred coordinates ('b')."""
    return _munk_slice("vb   3", alpha=(121, -20.3, 20.3), beta=(21, -8.0, 8.0), theta=[0.0, 2.0, 5.0],
                       nrz_range=(3, 800.0, 2800.0), rr_range=(4, 8.0, 26.0))


def munk3d_nx2d_v_gauss():
    """Nx2D 'v': arrivals and the eigen hits of each receiver bearing's plane."""
    return _munk_slice("vB   2", alpha=(121, -20.3, 20.3), theta=[0.0, 2.0, 5.0], nrz_range=(3, 800.0, 2800.0),
                       rr_range=(4, 8.0, 26.0))


CASES3D = {
    "munk3d_gauss": munk3d_gauss,
    "munk3d_hat": munk3d_hat,
    "munk3d_hat_incoherent": munk3d_hat_incoherent,
    "munk3d_gauss_semicoherent": munk3d_gauss_semicoherent,
    "munk3d_sources": munk3d_sources,
    "hex3d_gauss": hex3d_gauss,
    "seamount3d_gauss": seamount3d_gauss,
    "parabot3d_hat": parabot3d_hat,
    "munk3d_arr_gauss": munk3d_arr_gauss,
    "munk3d_arr_hat": munk3d_arr_hat,
    "parabot3d_arr_hat": parabot3d_arr_hat,
    "munk3d_eig_gauss": munk3d_eig_gauss,
    "seamount3d_eig_hat": seamount3d_eig_hat,
    "munk3d_brc_gauss": munk3d_brc_gauss,
    "munk3d_ray": munk3d_ray,
    "seamount3d_ray": seamount3d_ray,
    "munk3d_raycen_hat": munk3d_raycen_hat,
    "munk3d_raycen_gauss": munk3d_raycen_gauss,
    "seamount3d_raycen_hat": seamount3d_raycen_hat,
    "parabot3d_raycen_incoherent": parabot3d_raycen_incoherent,
    "munk3d_nx2d_gauss": munk3d_nx2d_gauss,
    "hex3d_nx2d_hat": hex3d_nx2d_hat,
    "seamount3d_nx2d_gauss": seamount3d_nx2d_gauss,
    "parabot3d_nx2d_incoherent": parabot3d_nx2d_incoherent,
    "parabot3d_curv_hat": parabot3d_curv_hat,
    "seamount3d_curv_gauss": seamount3d_curv_gauss,
    "parabot3d_curv_nx2d": parabot3d_curv_nx2d,
    "munk3d_nx2d_ray": munk3d_nx2d_ray,
    "seamount3d_nx2d_ray": seamount3d_nx2d_ray,
    "munk3d_nx2d_arr_gauss": munk3d_nx2d_arr_gauss,
    "munk3d_nx2d_eig_gauss": munk3d_nx2d_eig_gauss,
    "munk3d_raycen_arr_gauss": munk3d_raycen_arr_gauss,
    "munk3d_raycen_eig_hat": munk3d_raycen_eig_hat,
    "seamount3d_nx2d_arr_hat": seamount3d_nx2d_arr_hat,
    "munk3d_v_hat": munk3d_v_hat,
    "munk3d_raycen_v_gauss": munk3d_raycen_v_gauss,
    "munk3d_nx2d_v_gauss": munk3d_nx2d_v_gauss,
}
