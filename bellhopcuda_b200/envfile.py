"""Environment description and BELLHOP-format file writer (2-D).

An :class:`EnvSpec` holds the values an ``.env`` / ``.bty`` / ``.ati`` / ``.sbp``
file set carries, in the same units and with the same "sub-tabulation"
conventions as the reference's readers (reference: src/module/*.hpp Read
methods, src/api.cpp:253-277 for the read order). :func:`write_env` writes the
files; the product's native reader (``bhcb_setup_file``) and the reference's
``bellhopcxx`` both consume them, which is how parity runs feed identical
inputs to every implementation.

Numbers are written with ``repr`` (shortest round-trip text), so a reader using
``strtod`` recovers the exact double and one using ``strtof`` the correctly
rounded float, as the reference does for source/receiver depths
(include/bhc/structs.hpp:289-291).
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional, Sequence


def _num(v) -> str:
    if isinstance(v, (int,)) and not isinstance(v, bool):
        return str(v)
    return repr(float(v))


@dataclasses.dataclass
class EnvSpec:
    """One 2-D environment (a single ``.env`` plus optional side files)."""

    title: str = "bhcb env"
    freq: float = 50.0
    # TopOpt (module/topopt.hpp): SSP type, top BC, attenuation units, vol. atten
    ssp_type: str = "C"
    top_bc: str = "V"
    atten_unit: str = "W"
    vol_atten: str = " "
    single_beam: bool = False  # TopOpt[5] == 'I'
    # SSP nodes: z, cp, cs, rho, ap, as (module/ssp.hpp:74-118)
    ssp_z: Sequence[float] = (0.0, 5000.0)
    ssp_cp: Sequence[float] = (1500.0, 1500.0)
    ssp_cs: Optional[Sequence[float]] = None
    ssp_rho: Optional[Sequence[float]] = None
    ssp_ap: Optional[Sequence[float]] = None
    ssp_as: Optional[Sequence[float]] = None
    # halfspaces: zTemp alphaR betaR rho alphaI betaI (module/boundarycond.hpp:40-58)
    top_hs: Sequence[float] = (0.0, 1500.0, 0.0, 1.0, 0.0, 0.0)
    top_mz: float = 0.0
    bot_bc: str = "A"
    bot_hs: Sequence[float] = (5000.0, 1600.0, 0.0, 1.8, 0.8, 0.0)
    bot_mz: float = 0.0
    # Francois-Garrison: T S pH z_bar ; biological layers: (z1 z2 f0 q a0)
    fg: Sequence[float] = (20.0, 35.0, 8.0, 0.0)
    bio: Sequence[Sequence[float]] = ()
    # boundary files: ranges (km), depths (m), optional long-format geo rows
    bty_r: Optional[Sequence[float]] = None
    bty_z: Optional[Sequence[float]] = None
    bty_type: str = "LS"
    bty_geo: Optional[Sequence[Sequence[float]]] = None
    ati_r: Optional[Sequence[float]] = None
    ati_z: Optional[Sequence[float]] = None
    ati_type: str = "LS"
    ati_geo: Optional[Sequence[Sequence[float]]] = None
    # source beam pattern: (angle deg, level dB) pairs
    sbp: Optional[Sequence[Sequence[float]]] = None
    # vectors in file form: count + listed values (2 values + count => SubTab)
    nsz: int = 1
    sz: Sequence[float] = (1000.0,)
    nrz: int = 201
    rz: Sequence[float] = (0.0, 5000.0)
    nrr: int = 1001
    rr_km: Sequence[float] = (0.0, 100.0)
    run_type: str = "CG RR "
    nalpha: int = 2001
    isingle: int = 0
    alpha: Sequence[float] = (-20.0, 20.0)
    deltas: float = 0.0
    box_z: float = 5500.0
    box_r_km: float = 101.0

    @property
    def bot_depth(self) -> float:
        return float(self.ssp_z[-1])

    def ssp_cols(self) -> List[List[float]]:
        n = len(self.ssp_z)
        def col(v, d):
            return [float(x) for x in v] if v is not None else [d] * n
        return [
            [float(x) for x in self.ssp_z],
            [float(x) for x in self.ssp_cp],
            col(self.ssp_cs, 0.0),
            col(self.ssp_rho, 1.0),
            col(self.ssp_ap, 0.0),
            col(self.ssp_as, 0.0),
        ]


def env_text(spec: EnvSpec) -> str:
    """The ``.env`` file contents for ``spec``."""
    L: List[str] = []
    L.append("'%s'" % spec.title.replace("'", ""))
    L.append(_num(spec.freq))
    L.append("1")
    top_file = spec.ati_r is not None
    opt = (spec.ssp_type + spec.top_bc + spec.atten_unit + spec.vol_atten
           + ("~" if top_file else " ") + ("I" if spec.single_beam else " "))
    L.append("'%s'" % opt)
    if spec.vol_atten == "F":
        L.append(" ".join(_num(v) for v in spec.fg))
    elif spec.vol_atten == "B":
        L.append(str(len(spec.bio)))
        for b in spec.bio:
            L.append(" ".join(_num(v) for v in b))
    if spec.top_bc == "A":
        L.append(" ".join(_num(v) for v in spec.top_hs) + " /")
    elif spec.top_bc == "G":
        L.append(_num(spec.top_hs[0]) + " " + _num(spec.top_mz) + " /")
    z, cp, cs, rho, ap, as_ = spec.ssp_cols()
    L.append("%d 0.0 %s" % (len(z), _num(spec.bot_depth)))
    for i in range(len(z)):
        L.append("%s %s %s %s %s %s /" % (_num(z[i]), _num(cp[i]), _num(cs[i]),
                                          _num(rho[i]), _num(ap[i]), _num(as_[i])))
    bot_file = spec.bty_r is not None
    L.append("'%s%s' 0.0" % (spec.bot_bc, "~" if bot_file else " "))
    if spec.bot_bc == "A":
        L.append(" ".join(_num(v) for v in spec.bot_hs) + " /")
    elif spec.bot_bc == "G":
        L.append(_num(spec.bot_hs[0]) + " " + _num(spec.bot_mz) + " /")
    L.append(str(spec.nsz))
    L.append(" ".join(_num(v) for v in spec.sz) + " /")
    L.append(str(spec.nrz))
    L.append(" ".join(_num(v) for v in spec.rz) + " /")
    L.append(str(spec.nrr))
    L.append(" ".join(_num(v) for v in spec.rr_km) + " /")
    run = (spec.run_type + " " * 7)[:7]
    if spec.sbp is not None:  # source beam pattern file flag (module/sbp.hpp:35-38)
        run = run[:2] + "*" + run[3:]
    run = run.rstrip()
    L.append("'%s'" % run)
    if spec.single_beam:
        L.append("%d %d" % (spec.nalpha, spec.isingle))
    else:
        L.append(str(spec.nalpha))
    L.append(" ".join(_num(v) for v in spec.alpha) + " /")
    L.append("%s %s %s" % (_num(spec.deltas), _num(spec.box_z), _num(spec.box_r_km)))
    return "\n".join(L) + "\n"


def _bdry_text(btype: str, r, z, geo) -> str:
    L = ["'%s'" % btype, str(len(r))]
    for i in range(len(r)):
        row = [_num(r[i]), _num(z[i])]
        if btype[1:2] == "L" and geo is not None:
            row += [_num(v) for v in geo[i]]
        L.append(" ".join(row))
    return "\n".join(L) + "\n"


def write_env(spec: EnvSpec, fileroot: str) -> str:
    """Write ``fileroot``.env (+ .bty/.ati/.sbp when used). Returns fileroot."""
    d = os.path.dirname(fileroot)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(fileroot + ".env", "w") as f:
        f.write(env_text(spec))
    if spec.bty_r is not None:
        with open(fileroot + ".bty", "w") as f:
            f.write(_bdry_text(spec.bty_type, spec.bty_r, spec.bty_z, spec.bty_geo))
    if spec.ati_r is not None:
        with open(fileroot + ".ati", "w") as f:
            f.write(_bdry_text(spec.ati_type, spec.ati_r, spec.ati_z, spec.ati_geo))
    if spec.sbp is not None:
        with open(fileroot + ".sbp", "w") as f:
            f.write("%d\n" % len(spec.sbp))
            for a, db in spec.sbp:
                f.write("%s %s\n" % (_num(a), _num(db)))
    return fileroot
