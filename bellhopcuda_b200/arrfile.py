"""Readers for BELLHOP arrivals files (``.arr``): binary (RunType 'a') and
ASCII ('A').

Layout follows the reference writer (src/mode/arr.cpp:88-239): Fortran
sequential unformatted records ([int32 n][n bytes][int32 n]); a header of
'2D', freq, NSz+Sz, NRz+Rz, NRr+Rr, then per source the max arrival count
and, per receiver (depth-major, range fastest), the arrival count followed by
one record per arrival: a, phase (deg), delay (re, im), source and receiver
declination, top and bottom bounce counts (as floats).
"""
from __future__ import annotations

import numpy as np


def _records(raw: bytes):
    off = 0
    while off + 4 <= len(raw):
        n = int(np.frombuffer(raw, "<i4", 1, off)[0])
        yield raw[off + 4: off + 4 + n]
        off += n + 8


def read_arr_binary(path: str) -> dict:
    """2-D or 3-D binary arrivals. 3-D files add source x / y (m), receiver
    bearings (deg) and per arrival the source and receiver azimuths: records of
    10 floats (a, phase, delay re / im, src decl, src azim, rcvr decl, rcvr
    azim, top, bottom bounces) against 8 in 2-D. Receivers are listed per
    source as (bearing, depth, range), range fastest."""
    recs = _records(open(path, "rb").read())
    dim = next(recs)[:4].decode()
    is3d = "3" in dim
    freq = float(np.frombuffer(next(recs), "<f4", 1)[0])
    sx = sy = np.zeros(1)
    if is3d:
        r = next(recs); nsx = int(np.frombuffer(r, "<i4", 1)[0]); sx = np.frombuffer(r, "<f8", nsx, 4)
        r = next(recs); nsy = int(np.frombuffer(r, "<i4", 1)[0]); sy = np.frombuffer(r, "<f8", nsy, 4)
    r = next(recs); nsz = int(np.frombuffer(r, "<i4", 1)[0]); sz = np.frombuffer(r, "<f4", nsz, 4)
    r = next(recs); nrz = int(np.frombuffer(r, "<i4", 1)[0]); rz = np.frombuffer(r, "<f4", nrz, 4)
    r = next(recs); nrr = int(np.frombuffer(r, "<i4", 1)[0]); rr = np.frombuffer(r, "<f8", nrr, 4)
    theta = np.zeros(1)
    if is3d:
        r = next(recs); nth = int(np.frombuffer(r, "<i4", 1)[0]); theta = np.frombuffer(r, "<f8", nth, 4)
    nf = 10 if is3d else 8
    out = []
    for _src in range(nsz * len(sx) * len(sy)):
        maxn = int(np.frombuffer(next(recs), "<i4", 1)[0])
        src = []
        for _ in range(len(theta) * nrz * nrr):
            narr = int(np.frombuffer(next(recs), "<i4", 1)[0])
            arrs = [np.frombuffer(next(recs), "<f4", nf).copy() for _ in range(narr)]
            src.append(np.array(arrs, dtype=np.float32).reshape(narr, nf))
        out.append(dict(maxn=maxn, arrivals=src))
    return dict(dim=dim, freq=freq, sx=sx, sy=sy, sz=sz, rz=rz, rr=rr, theta=theta, sources=out)


def read_arr_ascii(path: str) -> dict:
    """2-D or 3-D ASCII arrivals (RunType 'A'), the same layout as the binary
    file as list-directed text: the dimension ('2D' / '3D'), the frequency,
    one line per coordinate array (count, values), then per source its
    largest arrival count and per receiver the count and one line per
    arrival. Returns the read_arr_binary dictionary (records as float32)."""
    lines = [ln.replace(",", " ").split() for ln in open(path) if ln.strip()]
    dim = "'" + lines[0][0].strip("'") + "'"
    is3d = "3" in dim
    freq = float(lines[1][0])
    k = 2

    def arr(dtype):
        nonlocal k
        n = int(lines[k][0])
        vals = [float(v) for v in lines[k][1:1 + n]]
        k += 1
        while len(vals) < n:   # a list-directed statement may continue on the next lines
            vals += [float(v) for v in lines[k]]
            k += 1
        return np.array(vals[:n], dtype)

    sx = sy = np.zeros(1)
    if is3d:
        sx, sy = arr(np.float64), arr(np.float64)
    sz, rz, rr = arr(np.float32), arr(np.float32), arr(np.float64)
    theta = arr(np.float64) if is3d else np.zeros(1)
    nf = 10 if is3d else 8
    out = []
    for _src in range(len(sz) * len(sx) * len(sy)):
        maxn = int(lines[k][0])
        k += 1
        src = []
        for _ in range(len(theta) * len(rz) * len(rr)):
            narr = int(lines[k][0])
            k += 1
            a = np.array([[float(v) for v in lines[k + j][:nf]] for j in range(narr)], np.float32)
            k += narr
            src.append(a.reshape(narr, nf))
        out.append(dict(maxn=maxn, arrivals=src))
    return dict(dim=dim, freq=freq, sx=sx, sy=sy, sz=sz, rz=rz, rr=rr, theta=theta, sources=out)
