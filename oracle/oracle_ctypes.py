"""ORACLE — test infrastructure only.

ctypes binding of the C restatement in oracle2d.c. Imported only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, and there only as the
checker. The product never imports this module.

``run(spec)`` takes a :class:`bellhopcuda_b200.envfile.EnvSpec`, converts its
file-level values exactly as the reference's list-directed reader would
(``strtod`` for doubles, ``strtof`` for the float depth vectors, the -999.9
sub-tabulation markers of src/common_setup.hpp:370-381) and runs the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle2d.so")

_libc = C.CDLL(None)
_libc.strtof.restype = C.c_float
_libc.strtof.argtypes = [C.c_char_p, C.c_void_p]
_libc.strtod.restype = C.c_double
_libc.strtod.argtypes = [C.c_char_p, C.c_void_p]


def _f32(v) -> float:
    return _libc.strtof(repr(float(v)).encode(), None)


def _f64(v) -> float:
    return _libc.strtod(repr(float(v)).encode(), None)


class O2Env(C.Structure):
    _fields_ = [
        ("run_type", C.c_char * 7), ("ssp_type", C.c_char), ("top_bc", C.c_char),
        ("atten_unit", C.c_char * 2), ("bot_bc", C.c_char), ("top_file", C.c_char),
        ("bot_file", C.c_char), ("freq0", C.c_double),
        ("fg_T", C.c_double), ("fg_S", C.c_double), ("fg_pH", C.c_double), ("fg_zbar", C.c_double),
        ("nbio", C.c_int32), ("bio", C.POINTER(C.c_double)),
        ("top_hs", C.c_double * 7), ("bot_hs", C.c_double * 7),
        ("nssp", C.c_int32),
        ("ssp_z", C.POINTER(C.c_double)), ("ssp_alphaR", C.POINTER(C.c_double)),
        ("ssp_betaR", C.POINTER(C.c_double)), ("ssp_rho", C.POINTER(C.c_double)),
        ("ssp_alphaI", C.POINTER(C.c_double)), ("ssp_betaI", C.POINTER(C.c_double)),
        ("bot_depth", C.c_double),
        ("top_type", C.c_char * 2), ("bot_type", C.c_char * 2),
        ("ntop", C.c_int32), ("nbot", C.c_int32),
        ("top_r", C.POINTER(C.c_double)), ("top_z", C.POINTER(C.c_double)),
        ("top_geo", C.POINTER(C.c_double)),
        ("bot_r", C.POINTER(C.c_double)), ("bot_z", C.POINTER(C.c_double)),
        ("bot_geo", C.POINTER(C.c_double)),
        ("nsbp", C.c_int32), ("sbp", C.POINTER(C.c_double)),
        ("nsz", C.c_int32), ("nrz", C.c_int32), ("nrr", C.c_int32), ("nalpha", C.c_int32),
        ("sz_in", C.POINTER(C.c_float)), ("rz_in", C.POINTER(C.c_float)),
        ("rr_in", C.POINTER(C.c_double)), ("alpha_in", C.POINTER(C.c_double)),
        ("isingle", C.c_int32), ("deltas", C.c_double), ("box_z", C.c_double),
        ("box_r_km", C.c_double),
        ("max_narr", C.c_int32), ("allow_merging", C.c_int32), ("eigen_memsize", C.c_int32),
    ]


class O2Arrival(C.Structure):
    _fields_ = [("NTopBnc", C.c_int32), ("NBotBnc", C.c_int32),
                ("SrcDeclAngle", C.c_float), ("SrcAzimAngle", C.c_float),
                ("RcvrDeclAngle", C.c_float), ("RcvrAzimAngle", C.c_float),
                ("a", C.c_float), ("Phase", C.c_float),
                ("delay_re", C.c_float), ("delay_im", C.c_float)]


ARRIVAL_DTYPE = np.dtype([("NTopBnc", "<i4"), ("NBotBnc", "<i4"), ("SrcDeclAngle", "<f4"),
                          ("SrcAzimAngle", "<f4"), ("RcvrDeclAngle", "<f4"),
                          ("RcvrAzimAngle", "<f4"), ("a", "<f4"), ("Phase", "<f4"),
                          ("delay_re", "<f4"), ("delay_im", "<f4")])
HIT_DTYPE = np.dtype([(k, "<i4") for k in ("is", "itheta", "ir", "iz", "isx", "isy", "isz",
                                           "ialpha", "ibeta")])


class O2Out(C.Structure):
    _fields_ = [
        ("NSz", C.c_int32), ("NRz", C.c_int32), ("NRz_per_range", C.c_int32),
        ("NRr", C.c_int32), ("Nalpha", C.c_int32),
        ("field", C.POINTER(C.c_float)), ("narr", C.POINTER(C.c_int32)),
        ("arr", C.c_void_p), ("hits", C.c_void_p), ("neigen", C.c_int32),
        ("rr_m", C.POINTER(C.c_double)), ("rz_m", C.POINTER(C.c_float)),
        ("alpha_rad", C.POINTER(C.c_double)),
        ("nsteps", C.c_int64), ("nevals", C.c_int64),
        ("err_bits", C.c_uint32), ("warn_bits", C.c_uint32),
        ("ray_first", C.c_int32), ("ray_count", C.c_int32),
    ]


_lib = None


def load():
    """Load (building if needed) the oracle shared library."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE])
        _lib = C.CDLL(LIB_PATH)
        _lib.oracle2d_run.argtypes = [C.POINTER(O2Env), C.POINTER(O2Out)]
        _lib.oracle2d_sizes.argtypes = [C.POINTER(O2Env), C.POINTER(O2Out)]
    return _lib


def _darr(vals):
    a = np.ascontiguousarray(np.array(vals, dtype=np.float64))
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _vec_in(n, vals, f32):
    """ReadVector semantics: max(3,n) slots, [1],[2] preset to -999.9f."""
    m = max(3, n)
    conv = _f32 if f32 else _f64
    out = [0.0] * m
    out[1] = out[2] = conv(-999.9) if f32 else float(np.float32(-999.9))
    for i, v in enumerate(vals[:n]):
        out[i] = conv(v)
    return out


class _Keep(list):
    pass


def make_env(spec, max_narr=20, allow_merging=1, eigen_memsize=100000):
    keep = _Keep()
    e = O2Env()
    rt = (spec.run_type + " " * 7)[:7]
    if spec.sbp is not None:
        rt = rt[:2] + "*" + rt[3:]
    e.run_type = rt.encode()
    e.ssp_type = spec.ssp_type.encode()
    e.top_bc = spec.top_bc.encode()
    e.atten_unit = (spec.atten_unit + spec.vol_atten).encode()
    e.bot_bc = spec.bot_bc.encode()
    e.top_file = b"~" if spec.ati_r is not None else b" "
    e.bot_file = b"~" if spec.bty_r is not None else b" "
    e.freq0 = _f64(spec.freq)
    e.fg_T, e.fg_S, e.fg_pH, e.fg_zbar = [_f64(v) for v in spec.fg]
    bio = [_f64(v) for b in spec.bio for v in b] or [0.0]
    a, p = _darr(bio); keep.append(a); e.bio = p; e.nbio = len(spec.bio)
    th = [_f64(v) for v in spec.top_hs] + [_f64(spec.top_mz)]
    bh = [_f64(v) for v in spec.bot_hs] + [_f64(spec.bot_mz)]
    e.top_hs = (C.c_double * 7)(*th)
    e.bot_hs = (C.c_double * 7)(*bh)
    cols = spec.ssp_cols()
    e.nssp = len(cols[0])
    names = ["ssp_z", "ssp_alphaR", "ssp_betaR", "ssp_rho", "ssp_alphaI", "ssp_betaI"]
    for nm, col in zip(names, cols):
        a, p = _darr([_f64(v) for v in col]); keep.append(a); setattr(e, nm, p)
    e.bot_depth = _f64(spec.bot_depth)
    for side in ("top", "bot"):
        r = spec.ati_r if side == "top" else spec.bty_r
        z = spec.ati_z if side == "top" else spec.bty_z
        g = spec.ati_geo if side == "top" else spec.bty_geo
        t = spec.ati_type if side == "top" else spec.bty_type
        setattr(e, side + "_type", t.encode())
        if r is None:
            r, z = [0.0], [0.0]
        a, p = _darr([_f64(v) for v in r]); keep.append(a); setattr(e, side + "_r", p)
        a, p = _darr([_f64(v) for v in z]); keep.append(a); setattr(e, side + "_z", p)
        geo = [_f64(v) for row in (g or []) for v in row] or [0.0]
        a, p = _darr(geo); keep.append(a); setattr(e, side + "_geo", p)
        setattr(e, "n" + side, len(r))
    if spec.sbp is not None:
        a, p = _darr([_f64(v) for row in spec.sbp for v in row]); keep.append(a)
        e.sbp = p; e.nsbp = len(spec.sbp)
    else:
        e.nsbp = 0
        a, p = _darr([0.0]); keep.append(a); e.sbp = p
    e.nsz, e.nrz, e.nrr, e.nalpha = spec.nsz, spec.nrz, spec.nrr, spec.nalpha
    sz = np.array(_vec_in(spec.nsz, list(spec.sz), True), dtype=np.float32)
    rz = np.array(_vec_in(spec.nrz, list(spec.rz), True), dtype=np.float32)
    rr = np.array(_vec_in(spec.nrr, list(spec.rr_km), False), dtype=np.float64)
    na = max(3, spec.nalpha, 2)
    al = [0.0] * na
    for i, v in enumerate(list(spec.alpha)[:max(spec.nalpha, 2)]):
        al[i] = _f64(v)
    if spec.nalpha > 2:
        al[2] = float(np.float32(-999.9))
    al = np.array(al, dtype=np.float64)
    keep += [sz, rz, rr, al]
    e.sz_in = sz.ctypes.data_as(C.POINTER(C.c_float))
    e.rz_in = rz.ctypes.data_as(C.POINTER(C.c_float))
    e.rr_in = rr.ctypes.data_as(C.POINTER(C.c_double))
    e.alpha_in = al.ctypes.data_as(C.POINTER(C.c_double))
    e.isingle = spec.isingle if spec.single_beam else 0
    e.deltas, e.box_z, e.box_r_km = _f64(spec.deltas), _f64(spec.box_z), _f64(spec.box_r_km)
    e.max_narr, e.allow_merging, e.eigen_memsize = max_narr, allow_merging, eigen_memsize
    return e, keep


def run(spec, max_narr=20, allow_merging=1, eigen_memsize=100000, rays=None):
    """Run the oracle; returns a dict with the scaled field / arrivals / hits."""
    lib = load()
    env, keep = make_env(spec, max_narr, allow_merging, eigen_memsize)
    out = O2Out()
    if lib.oracle2d_sizes(C.byref(env), C.byref(out)) != 0:
        raise RuntimeError("oracle: invalid environment")
    nsz, nrzp, nrr = out.NSz, out.NRz_per_range, out.NRr
    res = {"NSz": nsz, "NRz": out.NRz, "NRr": nrr, "Nalpha": out.Nalpha}
    rt = spec.run_type[0]
    field = narr = arr = hits = None
    if rt in "CSI":
        field = np.zeros((nsz, nrzp, nrr, 2), dtype=np.float32)
        out.field = field.ctypes.data_as(C.POINTER(C.c_float))
    if rt in "AaVv":
        narr = np.zeros((nsz, nrzp, nrr), dtype=np.int32)
        arr = np.zeros((nsz, nrzp, nrr, max_narr), dtype=ARRIVAL_DTYPE)
        out.narr = narr.ctypes.data_as(C.POINTER(C.c_int32))
        out.arr = arr.ctypes.data
    if rt in "EVv":
        hits = np.zeros(eigen_memsize, dtype=HIT_DTYPE)
        out.hits = hits.ctypes.data
    rr = np.zeros(nrr, np.float64)
    rz = np.zeros(out.NRz, np.float32)
    al = np.zeros(max(out.Nalpha, 1) + 4096, np.float64)
    out.rr_m = rr.ctypes.data_as(C.POINTER(C.c_double))
    out.rz_m = rz.ctypes.data_as(C.POINTER(C.c_float))
    out.alpha_rad = al.ctypes.data_as(C.POINTER(C.c_double))
    if rays is not None:
        out.ray_first, out.ray_count = rays
    rc = lib.oracle2d_run(C.byref(env), C.byref(out))
    del keep
    if field is not None:
        res["field"] = field[..., 0] + 1j * field[..., 1]
    if narr is not None:
        res["narr"], res["arr"] = narr, arr
    if hits is not None:
        res["hits"] = hits[: min(out.neigen, eigen_memsize)]
        res["neigen"] = out.neigen
    res.update(rr=rr, rz=rz, nsteps=out.nsteps, nevals=out.nevals,
               err_bits=out.err_bits, warn_bits=out.warn_bits, rc=rc)
    return res


def run_threaded(spec, nthreads=None, chunk=None):
    """Coherent TL of the whole fan, traced in ray ranges on host threads.

    The C restatement holds no global state and ctypes releases the GIL for
    the call, so ray ranges run side by side; ScalePressure is linear for
    coherent runs, so the range fields add up to the field of the whole fan
    (float additions in another order: equal to within float rounding).
    Returns the summed field and the summed step and contribution counts."""
    from concurrent.futures import ThreadPoolExecutor
    if spec.run_type[0] != "C":
        raise ValueError("run_threaded: coherent TL runs only (incoherent fields are not additive)")
    n = sizes(spec)["Nalpha"]
    nthreads = nthreads or os.cpu_count() or 1
    chunk = chunk or max(1, -(-n // (4 * nthreads)))
    ranges = [(a, min(chunk, n - a)) for a in range(0, n, chunk)]
    with ThreadPoolExecutor(max_workers=nthreads) as ex:
        parts = list(ex.map(lambda r: run(spec, rays=r), ranges))
    out = dict(parts[0])
    out["field"] = sum(p["field"] for p in parts)
    out["nsteps"] = sum(p["nsteps"] for p in parts)
    out["nevals"] = sum(p["nevals"] for p in parts)
    out["err_bits"] = 0
    for p in parts:
        out["err_bits"] |= p["err_bits"]
    return out


def sizes(spec):
    """NSz, NRz, NRr and Nalpha as the oracle's preprocessing gives them."""
    lib = load()
    env, keep = make_env(spec)
    out = O2Out()
    if lib.oracle2d_sizes(C.byref(env), C.byref(out)) != 0:
        raise RuntimeError("oracle: invalid environment")
    del keep
    return {"NSz": out.NSz, "NRz": out.NRz, "NRz_per_range": out.NRz_per_range, "NRr": out.NRr,
            "Nalpha": out.Nalpha}


def reference_dir() -> str:
    """The reference source tree: $BHCB_REFERENCE, else oracle/Makefile's REF
    default (the one place that names it)."""
    env = os.environ.get("BHCB_REFERENCE")
    if env:
        return env
    try:
        return subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True,
                              check=True).stdout.strip()
    except (OSError, subprocess.CalledProcessError):
        return ""
