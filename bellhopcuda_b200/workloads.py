"""Seeded synthetic workloads (2-D) used by the tests and the benchmark.

No public dataset is involved: every environment is generated from a numpy
PCG64 seed, written as ordinary BELLHOP input files, and fed identically to
the reference, the oracle and this library.

* ``munk_tl``   — deep-water Munk profile, coherent hat-beam TL
                  (51 c-linear nodes, 2001 rays, 201 x 1001 receivers).
* ``rd_gauss``  — range-dependent Gaussian-beam TL: PCHIP Munk + smoothed
                  N(0, 2 m/s) perturbation on 64 nodes, 200-point bathymetry
                  uniform in 3000-5000 m over 100 km, 10 log-spaced frequencies
                  50-500 Hz, 20001 rays over +-30 deg, 501 x 2001 receivers.
* ``batch_envs`` — many small uneven spline-SSP environments for batched runs.
* ``c5_envs``   — surrogate training / test environments: 2-D coherent hat-beam
                  TL on a 128 x 256 grid; 64-node SSP = Munk + 8 random smooth
                  modes N(0, 2 m/s), depth 1000-5000 m, bottom cp 1500-1800
                  m/s, source 10-500 m, 50-500 Hz (log-uniform).
* ``c4_3d``     — 3-D Gaussian-beam TL (or arrivals): hexahedral SSP on a
                  41 x 41 x 51 grid over 80 x 80 km x 5000 m (Munk plus a seeded
                  warm-core eddy), 'R' bathymetry on a 101 x 101 grid seeded in
                  3000-5000 m, source 500 m, 200 Hz, 144 bearings x 361
                  elevations, receivers 36 bearings x 101 depths x 501 ranges.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from .envfile import EnvSpec
from . import envfile3d


def munk_c(z, eps=0.00737):
    """Canonical Munk profile c(z) = 1500 (1 + eps (eta - 1 + exp(-eta)))."""
    z = np.asarray(z, dtype=np.float64)
    eta = 2.0 * (z - 1300.0) / 1300.0
    return 1500.0 * (1.0 + eps * (eta - 1.0 + np.exp(-eta)))


def munk_tl(nalpha=2001, nrz=201, nrr=1001, freq=50.0, beam="G") -> EnvSpec:
    z = np.arange(0.0, 5000.0 + 1e-9, 100.0)
    return EnvSpec(
        title="Munk coherent TL", freq=freq, ssp_type="C", top_bc="V", atten_unit="W",
        ssp_z=z, ssp_cp=munk_c(z), bot_bc="A", bot_hs=(5000.0, 1600.0, 0.0, 1.8, 0.8, 0.0),
        nsz=1, sz=(1000.0,), nrz=nrz, rz=(0.0, 5000.0), nrr=nrr, rr_km=(0.0, 100.0),
        run_type="C%s RR " % beam, nalpha=nalpha, alpha=(-20.0, 20.0), deltas=0.0,
        box_z=5500.0, box_r_km=101.0)


def rd_gauss_freqs(n=10):
    return [float(f) for f in np.logspace(math.log10(50.0), math.log10(500.0), n)]


def rd_gauss(seed=1002, freq=None, nalpha=20001, nrz=501, nrr=2001, nbty=200) -> EnvSpec:
    """Range-dependent Gaussian-beam case; ``freq`` None -> the first frequency."""
    rng = np.random.Generator(np.random.PCG64(seed))
    z = np.linspace(0.0, 5000.0, 64)
    pert = rng.normal(0.0, 2.0, z.size)
    k = np.exp(-0.5 * (np.arange(-2, 3) / 1.0) ** 2)
    k /= k.sum()
    pert = np.convolve(np.pad(pert, 2, mode="edge"), k, mode="valid")
    c = munk_c(z) + pert
    br = np.linspace(0.0, 100.0, nbty)
    bz = rng.uniform(3000.0, 5000.0, nbty)
    zmax = float(bz.max())
    # the SSP must reach the deepest bathymetry point (module/boundary.hpp:419-425)
    z = z * (zmax / 5000.0)
    return EnvSpec(
        title="range-dependent Gaussian TL", freq=rd_gauss_freqs()[0] if freq is None else freq,
        ssp_type="P", top_bc="V", atten_unit="W", ssp_z=z, ssp_cp=c, bot_bc="A",
        bot_hs=(zmax, 1600.0, 0.0, 1.8, 0.8, 0.0), bty_r=br, bty_z=bz, bty_type="LS",
        nsz=1, sz=(1000.0,), nrz=nrz, rz=(0.0, zmax), nrr=nrr, rr_km=(0.0, 100.0),
        run_type="CB RR ", nalpha=nalpha, alpha=(-30.0, 30.0), deltas=0.0,
        box_z=zmax + 500.0, box_r_km=101.0)


def batch_envs(n=256, seed=1003, scale=1.0) -> List[EnvSpec]:
    """Uneven spline-SSP environments; ``scale`` < 1 shrinks rays/receivers."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        nn = int(rng.integers(20, 201))
        depth = float(rng.uniform(200.0, 5000.0))
        z = np.linspace(0.0, depth, nn)
        c = munk_c(z) + rng.normal(0.0, 3.0, nn)
        cp = float(rng.uniform(1500.0, 1800.0))
        rho = float(rng.uniform(1.5, 2.0))
        f = float(math.exp(rng.uniform(math.log(25.0), math.log(1000.0))))
        na = max(16, int(int(rng.integers(500, 20001)) * scale))
        nrz = max(8, int(int(rng.integers(100, 501)) * scale))
        nrr = max(8, int(int(rng.integers(200, 2001)) * scale))
        rmax = float(rng.uniform(10.0, 100.0))
        out.append(EnvSpec(
            title="batch env %d" % i, freq=f, ssp_type="S", top_bc="V", atten_unit="W",
            ssp_z=z, ssp_cp=c, bot_bc="A", bot_hs=(depth, cp, 0.0, rho, 0.5, 0.0),
            nsz=1, sz=(float(rng.uniform(0.05, 0.95)) * depth,), nrz=nrz, rz=(0.0, depth),
            nrr=nrr, rr_km=(0.0, rmax), run_type="CB RR ", nalpha=na, alpha=(-30.0, 30.0),
            deltas=0.0, box_z=depth + 100.0, box_r_km=rmax + 1.0))
    return out


def _smooth2d(a, sigma):
    """Separable Gaussian smoothing with reflecting edges."""
    r = int(math.ceil(3 * sigma))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    k /= k.sum()
    for ax in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[ax] = (r, r)
        b = np.pad(a, pad, mode="reflect")
        a = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), ax, b)
    return a


def c4_3d(seed=1004, run_type="CB   3", scale=1.0, nalpha=361, nbeta=144, ntheta=36, nrz=101, nrr=501,
          freq=200.0, step=100.0):
    """The 3-D workload as {suffix: file text}. ``scale`` < 1 shrinks the ray
    fan and the receiver grid (for parity cases); the environment is the same."""
    rng = np.random.Generator(np.random.PCG64(seed))
    # hexahedral SSP: Munk + warm-core eddy (+10 m/s, radius 20 km, depth scale 800 m)
    hx = np.linspace(-40.0, 40.0, 41)
    hy = np.linspace(-40.0, 40.0, 41)
    hz = np.linspace(0.0, 5000.0, 51)
    ex, ey = rng.uniform(-20.0, 20.0, 2)
    X, Y, Z = np.meshgrid(hx, hy, hz, indexing="ij")
    r2 = (X - ex) ** 2 + (Y - ey) ** 2
    c = munk_c(Z) + 10.0 * np.exp(-r2 / (2.0 * 20.0 ** 2)) * np.exp(-Z / 800.0)
    # bathymetry: U(3000, 5000) smoothed, rescaled back to 3000-5000 m
    bx = np.linspace(-40.0, 40.0, 101)
    by = np.linspace(-40.0, 40.0, 101)
    b = _smooth2d(rng.uniform(3000.0, 5000.0, (101, 101)), 4.0)
    b = 3000.0 + 2000.0 * (b - b.min()) / (b.max() - b.min())
    na = max(3, int(round(nalpha * scale)) | 1)
    nb = max(4, int(round(nbeta * scale)))
    env = envfile3d.env_text(
        title="3-D hexahedral Munk + eddy, gridded bathymetry", freq=freq, ssp_opt="HVW", depth=5000.0,
        ssp=[(float(z), float(munk_c(z))) for z in hz], bot=("A~", 1600.0, 1.8, 0.8), sx=[0.0], sy=[0.0],
        sz=[500.0], rz=None, rr_km=None, theta=None, run_type=run_type, alpha=(na, -30.0, 30.0),
        beta=(nb + 1, 0.0, 360.0), step=step, box_km=(39.0, 39.0), box_z=5100.0,
        nrz_range=(max(2, int(round(nrz * scale))), 0.0, 5000.0),
        rr_range=(max(2, int(round(nrr * scale))), 0.0, 38.0),
        theta_range=(max(1, int(round(ntheta * scale))), 0.0, 360.0 - 360.0 / max(1, int(round(ntheta * scale)))))
    return {".env": env, ".ssp": envfile3d.hex_ssp_text(hx, hy, hz, c), ".bty": envfile3d.grid_text(bx, by, b)}


C5_NZ, C5_NR = 128, 256
C5_RR_KM = (0.08, 20.0)
# launch angles -89 .. 89 degrees: the fan reaches every receiver of the grid
# (with -60 .. 60 a cone beside the source that no ray enters stays at the
# 130 dB clamp, up to 90 % of the first 300 m of range)
C5_FAN_DEG = 89.0


def c5_params(n, seed=1005, run_type="IB", fan_deg=C5_FAN_DEG):
    """Seeded parameters of n surrogate environments (one row each):
    depth, bottom cp, source depth, frequency, 8 SSP mode amplitudes; and
    the RunType of their fields ('IB': incoherent Gaussian beams, the
    default; 'CG': coherent hat beams) and the launch fan's half-angle."""
    rng = np.random.Generator(np.random.PCG64(seed))
    depth = rng.uniform(1000.0, 5000.0, n)
    cp = rng.uniform(1500.0, 1800.0, n)
    zs = rng.uniform(10.0, 500.0, n)
    f = np.exp(rng.uniform(math.log(50.0), math.log(500.0), n))
    a = rng.normal(0.0, 2.0, (n, 8))
    return dict(depth=depth, cp=cp, zs=zs, f=f, a=a, run_type=run_type, fan_deg=float(fan_deg))


def c5_ssp(depth, a):
    """64-node SSP: Munk + sum_k a_k sin(k pi z / D)."""
    z = np.linspace(0.0, depth, 64)
    c = munk_c(z) + sum(a[k] * np.sin((k + 1) * np.pi * z / depth) for k in range(8))
    return z, c


def c5_nalpha(depth, freq):
    """EstimateNumAngles (src/module/rayangles.hpp:212-238) for this grid."""
    rmax = C5_RR_KM[1] * 1000.0
    n = max(int(0.3 * rmax * freq / 1500.0), 300)
    return max(int(np.pi / np.arctan(depth / (10.0 * rmax))), n)


def c5_env(P, i) -> EnvSpec:
    depth, cp, zs, f = float(P["depth"][i]), float(P["cp"][i]), float(P["zs"][i]), float(P["f"][i])
    z, c = c5_ssp(depth, P["a"][i])
    return EnvSpec(
        title="surrogate env %d" % i, freq=f, ssp_type="C", top_bc="V", atten_unit="W",
        ssp_z=z, ssp_cp=c, bot_bc="A", bot_hs=(depth, cp, 0.0, 1.8, 0.8, 0.0),
        nsz=1, sz=(zs,), nrz=C5_NZ, rz=(0.0, depth), nrr=C5_NR, rr_km=C5_RR_KM,
        run_type=P.get("run_type", "IB")[:2] + " RR ", nalpha=c5_nalpha(depth, f),
        alpha=(-P.get("fan_deg", C5_FAN_DEG), P.get("fan_deg", C5_FAN_DEG)), deltas=0.0,
        box_z=depth + 100.0, box_r_km=C5_RR_KM[1] + 1.0)


def c5_envs(n=100000, seed=1005, run_type="IB") -> List[EnvSpec]:
    P = c5_params(n, seed, run_type)
    return [c5_env(P, i) for i in range(n)]
