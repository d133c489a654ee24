"""Reader for binary BELLHOP arrivals files (``.arr`` written for RunType 'a').

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
    recs = _records(open(path, "rb").read())
    dim = next(recs)[:4].decode()
    freq = float(np.frombuffer(next(recs), "<f4", 1)[0])
    r = next(recs); nsz = int(np.frombuffer(r, "<i4", 1)[0]); sz = np.frombuffer(r, "<f4", nsz, 4)
    r = next(recs); nrz = int(np.frombuffer(r, "<i4", 1)[0]); rz = np.frombuffer(r, "<f4", nrz, 4)
    r = next(recs); nrr = int(np.frombuffer(r, "<i4", 1)[0]); rr = np.frombuffer(r, "<f8", nrr, 4)
    out = []
    for _isz in range(nsz):
        maxn = int(np.frombuffer(next(recs), "<i4", 1)[0])
        src = []
        for _ in range(nrz * nrr):
            narr = int(np.frombuffer(next(recs), "<i4", 1)[0])
            arrs = [np.frombuffer(next(recs), "<f4", 8).copy() for _ in range(narr)]
            src.append(np.array(arrs, dtype=np.float32).reshape(narr, 8))
        out.append(dict(maxn=maxn, arrivals=src))
    return dict(dim=dim, freq=freq, sz=sz, rz=rz, rr=rr, sources=out)
