"""Reader for BELLHOP ``.shd`` shade files (TL output).

Layout follows the reference writer (src/mode/tl.cpp:38-101 header,
src/mode/tl.cpp:195-248 records): fixed-length records of ``LRecl`` 4-byte
words; record 0 holds LRecl and the title, records 2-9 the sizes and
coordinate vectors, and record ``10 + ((((isx*NSy+isy)*Ntheta+itheta)*NSz+isz)
*NRz_per_range + irz)`` holds ``NRr`` complex64 pressures.
"""
from __future__ import annotations

import numpy as np


def read_shd(path: str) -> dict:
    raw = open(path, "rb").read()
    lrecl = int(np.frombuffer(raw, "<i4", 1, 0)[0]) * 4

    def rec(i):
        return raw[i * lrecl:(i + 1) * lrecl]

    title = rec(0)[4:84].decode("latin1").rstrip()
    plot_type = rec(1)[:10].decode("latin1")
    r2 = rec(2)
    nfreq, ntheta, nsx, nsy, nsz, nrz, nrr = np.frombuffer(r2, "<i4", 7, 0)
    freq0, atten = np.frombuffer(r2, "<f8", 2, 28)
    freqs = np.frombuffer(rec(3), "<f8", nfreq)
    theta = np.frombuffer(rec(4), "<f8", ntheta)
    sz = np.frombuffer(rec(7), "<f4", nsz)
    rz = np.frombuffer(rec(8), "<f4", nrz)
    rr = np.frombuffer(rec(9), "<f8", nrr)
    nrzp = 1 if plot_type.startswith("irregular") else int(nrz)
    field = np.zeros((nsx, nsy, ntheta, nsz, nrzp, nrr), np.complex64)
    k = 10
    for isx in range(nsx):
        for isy in range(nsy):
            for it in range(ntheta):
                for isz in range(nsz):
                    for irz in range(nrzp):
                        field[isx, isy, it, isz, irz] = np.frombuffer(rec(k), "<c8", nrr)
                        k += 1
    return dict(title=title, plot_type=plot_type, freq0=float(freq0), atten=float(atten),
                freqs=freqs, theta=theta, sz=sz, rz=rz, rr=rr, field=field)
