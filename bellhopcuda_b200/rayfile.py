"""Reader for BELLHOP ``.ray`` files (ray trajectories, RunType 'R', and
eigenrays, 'E').

Layout follows the reference writer (src/mode/ray.hpp:176-247): a header of
title, frequency, NSx NSy NSz, Nalpha Nbeta, top depth, bottom depth and the
coordinate kind ('rz' or 'xyz'), then per ray its take-off angle, the number
of points with the top and bottom bounce counts of the last point, and one
line per point. Numbers are read as list-directed text, so files written by
the reference and by this library parse alike.
"""
from __future__ import annotations

import numpy as np


def read_ray(path: str) -> dict:
    lines = [ln.strip() for ln in open(path) if ln.strip()]
    title = lines[0].strip("'")
    freq = float(lines[1].split()[0])
    nsx, nsy, nsz = (int(v) for v in lines[2].split()[:3])
    nalpha, nbeta = (int(v) for v in lines[3].split()[:2])
    top, bot = float(lines[4].split()[0]), float(lines[5].split()[0])
    kind = lines[6].strip("'").strip()
    ncoord = 3 if kind == "xyz" else 2
    rays = []
    k = 7
    while k < len(lines):
        alpha = float(lines[k].split()[0])
        n, ntop, nbot = (int(float(v)) for v in lines[k + 1].split()[:3])
        pts = np.array([[float(v) for v in lines[k + 2 + j].split()[:ncoord]] for j in range(n)])
        rays.append(dict(alpha=alpha, ntop=ntop, nbot=nbot, xy=pts.reshape(n, ncoord)))
        k += 2 + n
    return dict(title=title, freq=freq, nsx=nsx, nsy=nsy, nsz=nsz, nalpha=nalpha, nbeta=nbeta,
                top=top, bot=bot, kind=kind, rays=rays)
