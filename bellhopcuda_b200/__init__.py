"""bellhopcuda_b200 — B200-native BELLHOP beam tracer (2-D field modes).

Python mirror of the reference's library flow (include/bhc/bhc.hpp):

    bhc::setup(init, params, outputs)   ->  Tracer(...).setup(file_root)
    bhc::run(params, outputs)           ->  Tracer.run()
    outputs.uAllSources                 ->  Tracer.field(env, ifreq)
    bhc::writeout(params, outputs, fr)  ->  Tracer.writeout(file_root)
    bhc::finalize(params, outputs)      ->  Tracer.close()

All compute happens in libbhcb.so (hand-written sm_100a kernels) through the C
ABI declared in include/bhcb.h. There is no CPU fallback: if the native
library is missing or no GPU is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbhcb.so")

PREC_FP64 = 0
PREC_MIXED = 1
FLAG_SERIAL_INFLUENCE = 1   # BHCB_FLAG_SERIAL_INFLUENCE (the default)
FLAG_OVERLAP_INFLUENCE = 2  # BHCB_FLAG_OVERLAP_INFLUENCE
FLAG_NO_GRAPH = 4           # BHCB_FLAG_NO_GRAPH
FLAG_PIPELINE = 8           # BHCB_FLAG_PIPELINE

ERR_NAMES = {
    2: "BHC_ERR_RAYINIT", 3: "BHC_ERR_BOUNDARY_SEG_CONTAINS_NAN",
    4: "BHC_ERR_BOUNDARY_CONDITION_TYPE", 5: "BHC_ERR_INVALID_SSP_TYPE",
    6: "BHC_ERR_OUTSIDE_ALTIMETRY", 7: "BHC_ERR_OUTSIDE_BATHYMETRY", 8: "BHC_ERR_OUTSIDE_SSP",
    9: "BHC_ERR_QUAD_ISEG", 31: "segment buffer overflow",
}


class BhcbError(RuntimeError):
    def __init__(self, code: int, msg: str, err_bits: int = 0):
        super().__init__("bhcb error %d: %s" % (code, msg))
        self.code = code
        self.err_bits = err_bits


class Tuning(C.Structure):
    _fields_ = [("trace_block", C.c_int32), ("influence_ctas_per_sm", C.c_int32), ("stage_kb", C.c_int32),
                ("trace_ms", C.c_double), ("influence_ms", C.c_double), ("trace_lanes", C.c_int32)]


class Init(C.Structure):
    _fields_ = [("gpu_index", C.c_int32), ("precision", C.c_int32), ("max_memory", C.c_uint64),
                ("share_trajectory", C.c_int32), ("flags", C.c_int32),
                ("output_callback", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("steps", C.c_uint64), ("segments", C.c_uint64),
                ("evals", C.c_uint64), ("err_bits", C.c_uint32), ("warn_bits", C.c_uint32),
                ("groups", C.c_int32), ("fields", C.c_int32), ("trace_ms", C.c_double),
                ("influence_ms", C.c_double), ("total_ms", C.c_double), ("h2d_bytes", C.c_uint64),
                ("influence_span_ms", C.c_double)]


class EnvInfo(C.Structure):
    _fields_ = [("nsz", C.c_int32), ("nrz", C.c_int32), ("nrz_per_range", C.c_int32),
                ("nrr", C.c_int32), ("nalpha", C.c_int32), ("ssp_type", C.c_int32),
                ("freq", C.c_double), ("deltas", C.c_double), ("run_type", C.c_char * 8),
                ("beam_type", C.c_char * 8)]


_PD = C.POINTER(C.c_double)
_PF = C.POINTER(C.c_float)


class EnvDesc(C.Structure):
    """bhcb_env_desc: a 2-D environment in memory (the values bhcParams<false>
    holds after bhc::setup, include/bhc/bhc.hpp:58-452)."""
    _fields_ = [("title", C.c_char_p), ("freq0", C.c_double), ("top_opt", C.c_char * 6),
                ("bot_opt", C.c_char * 6), ("fg", C.c_double * 4), ("nbio", C.c_int32), ("bio", _PD),
                ("top_hs", C.c_double * 7), ("bot_hs", C.c_double * 7), ("nssp", C.c_int32),
                ("ssp_z", _PD), ("ssp_alphaR", _PD), ("ssp_betaR", _PD), ("ssp_rho", _PD),
                ("ssp_alphaI", _PD), ("ssp_betaI", _PD), ("bot_depth", C.c_double),
                ("ati_type", C.c_char * 2), ("bty_type", C.c_char * 2), ("nati", C.c_int32),
                ("nbty", C.c_int32), ("ati_r_km", _PD), ("ati_z", _PD), ("ati_geo", _PD),
                ("bty_r_km", _PD), ("bty_z", _PD), ("bty_geo", _PD), ("nsbp", C.c_int32), ("sbp", _PD),
                ("nsz", C.c_int32), ("nrz", C.c_int32), ("nrr", C.c_int32), ("nalpha", C.c_int32),
                ("isingle", C.c_int32), ("sz", _PF), ("rz", _PF), ("rr_km", _PD), ("alpha_deg", _PD),
                ("run_type", C.c_char * 7), ("cerv_type", C.c_char * 2), ("deltas", C.c_double),
                ("box_z", C.c_double), ("box_r_km", C.c_double), ("eps_mult", C.c_double),
                ("rloop", C.c_double), ("nimage", C.c_int32), ("ibeam_window", C.c_int32),
                ("component", C.c_char), ("nquad_r", C.c_int32), ("quad_r_km", _PD), ("quad_c", _PD),
                ("nbrc", C.c_int32), ("ntrc", C.c_int32), ("brc", _PD), ("trc", _PD)]


# bhcb_arrival / bhcb_eigen_hit (the reference's Arrival and EigenHit records)
ARRIVAL_DTYPE = np.dtype([("NTopBnc", "<i4"), ("NBotBnc", "<i4"), ("SrcDeclAngle", "<f4"),
                          ("SrcAzimAngle", "<f4"), ("RcvrDeclAngle", "<f4"), ("RcvrAzimAngle", "<f4"),
                          ("a", "<f4"), ("Phase", "<f4"), ("delay_re", "<f4"), ("delay_im", "<f4")])
EIGEN_HIT_DTYPE = np.dtype([(n, "<i4") for n in ("is", "itheta", "ir", "iz", "isx", "isy", "isz",
                                                 "ialpha", "ibeta")])

_lib = None

# (name, restype, argtypes) for every entry point of include/bhcb.h
SIGNATURES = [
    ("bhcb_open", C.c_int, [C.POINTER(Init), C.POINTER(C.c_void_p)]),
    ("bhcb_close", None, [C.c_void_p]),
    ("bhcb_setup", C.c_int, [C.c_void_p, C.c_char_p]),
    ("bhcb_add_env", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32)]),
    ("bhcb_clear", C.c_int, [C.c_void_p]),
    ("bhcb_set_frequencies", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    ("bhcb_run", C.c_int, [C.c_void_p]),
    ("bhcb_prepare", C.c_int, [C.c_void_p]),
    ("bhcb_launch", C.c_int, [C.c_void_p]),
    ("bhcb_sync", C.c_int, [C.c_void_p]),
    ("bhcb_field_shape", C.c_int, [C.c_void_p, C.c_int32] + [C.POINTER(C.c_int32)] * 4),
    ("bhcb_copy_field", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t]),
    ("bhcb_field_device", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    ("bhcb_receivers", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_int32,
                                 C.POINTER(C.c_float), C.c_int32]),
    ("bhcb_writeout", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_char_p]),
    ("bhcb_get_stats", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("bhcb_last_error", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32)]),
    ("bhcb_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("bhcb_run_noalloc", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t,
                                   C.c_char_p, C.c_size_t]),
    ("bhcb_check_env", C.c_int, [C.c_char_p, C.POINTER(EnvInfo), C.c_char_p, C.c_size_t]),
    ("bhcb_set_arrival_options", C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    ("bhcb_arrivals_shape", C.c_int, [C.c_void_p, C.c_int32, C.c_int32] + [C.POINTER(C.c_int32)] * 4),
    ("bhcb_copy_arrivals", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p,
                                     C.c_size_t]),
    ("bhcb_eigen_hits", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64,
                                  C.POINTER(C.c_int64)]),
    ("bhcb_check_env3d", C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.c_char_p,
                                   C.c_size_t]),
    ("bhcb_setup3d", C.c_int, [C.c_void_p, C.c_char_p]),
    ("bhcb_add_env3d", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32)]),
    ("bhcb_field_shape3d", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("bhcb_grid3d", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p]),
    ("bhcb_graph_create", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t,
                                    C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    ("bhcb_graph_launch", C.c_int, [C.c_void_p, C.c_void_p]),
    ("bhcb_graph_status", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    ("bhcb_graph_destroy", None, [C.c_void_p]),
    ("bhcb_nn_gemm", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("bhcb_nn_status", C.c_int, [C.POINTER(C.c_int32), C.c_int32]),
    ("bhcb_nn_tl_db", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float, C.c_void_p]),
    ("bhcb_nn_transpose", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    ("bhcb_nn_mse", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("bhcb_nn_row_rms", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    ("bhcb_nn_colsum", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    ("bhcb_nn_adam", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_float,
                               C.c_float, C.c_float, C.c_float, C.c_int32, C.c_float, C.c_void_p, C.c_void_p,
                               C.c_void_p]),
    ("bhcb_nn_to_bf16", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    ("bhcb_nn_affine", C.c_int, [C.c_void_p, C.c_int64, C.c_float, C.c_float, C.c_void_p]),
    ("bhcb_rays_shape", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("bhcb_copy_rays", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_size_t]),
    ("bhcb_autotune", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Tuning)]),
    ("bhcb_set_tuning", C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    ("bhcb_version", C.c_char_p, []),
    ("bhcb_add_env_desc", C.c_int, [C.c_void_p, C.POINTER(EnvDesc), C.POINTER(C.c_int32)]),
    ("bhcb_read_env_desc", C.c_int, [C.c_char_p, C.POINTER(C.POINTER(EnvDesc)), C.c_char_p, C.c_size_t]),
    ("bhcb_free_env_desc", None, [C.POINTER(EnvDesc)]),
    ("bhcb_ssp_at", C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.POINTER(C.c_double)]),
]


def load_library():
    """Load libbhcb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbhcb.so is missing: run `python -m bellhopcuda_b200.build` "
                               "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class EnvDescription:
    """An environment read into memory by the library (bhcb_read_env_desc):
    `desc` is the EnvDesc, editable in place (scalars; the arrays stay the
    library's); released with close() or on garbage collection."""

    def __init__(self, file_root: str):
        lib = load_library()
        p = C.POINTER(EnvDesc)()
        msg = C.create_string_buffer(512)
        rc = lib.bhcb_read_env_desc(file_root.encode(), C.byref(p), msg, 512)
        if rc != 0:
            raise BhcbError(rc, msg.value.decode(errors="replace"))
        self._p = p
        self.desc = p.contents

    def close(self):
        if self._p:
            load_library().bhcb_free_env_desc(self._p)
            self._p = None
            self.desc = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def check_env(file_root: str) -> dict:
    """Read and validate an environment on the host only (no GPU needed)."""
    lib = load_library()
    info = EnvInfo()
    msg = C.create_string_buffer(512)
    rc = lib.bhcb_check_env(file_root.encode(), C.byref(info), msg, 512)
    if rc != 0:
        raise BhcbError(rc, msg.value.decode(errors="replace"))
    return dict(nsz=info.nsz, nrz=info.nrz, nrz_per_range=info.nrz_per_range, nrr=info.nrr,
                nalpha=info.nalpha, ssp_type=info.ssp_type, freq=info.freq, deltas=info.deltas,
                run_type=info.run_type.decode(), beam_type=info.beam_type.decode())


def check_env3d(file_root: str) -> dict:
    """Validate a 3-D environment on the host (no GPU): field dims and ray count."""
    lib = load_library()
    dims = (C.c_int32 * 6)()
    nrays = C.c_int64()
    msg = C.create_string_buffer(512)
    rc = lib.bhcb_check_env3d(file_root.encode(), dims, C.byref(nrays), msg, len(msg))
    if rc != 0:
        raise BhcbError(rc, msg.value.decode(errors="replace"))
    return {"dims": tuple(int(d) for d in dims), "nrays": nrays.value}


class Tracer:
    """One bhcb context (one GPU, one stream)."""

    def __init__(self, gpu: int = 0, precision: int = PREC_MIXED, max_memory: int = 0,
                 share_trajectory: bool = True, serial_influence: bool = False, overlap_influence: bool = False,
                 graphs: bool = True, pipeline: bool = False):
        self._lib = load_library()
        flags = (FLAG_SERIAL_INFLUENCE if serial_influence else 0) | \
            (FLAG_OVERLAP_INFLUENCE if overlap_influence else 0) | (0 if graphs else FLAG_NO_GRAPH) | \
            (FLAG_PIPELINE if pipeline else 0)
        init = Init(gpu, precision, max_memory, 1 if share_trajectory else 0, flags, None)
        h = C.c_void_p()
        rc = self._lib.bhcb_open(C.byref(init), C.byref(h))
        if rc != 0:
            raise BhcbError(rc, "bhcb_open failed (no usable CUDA device?)")
        self._h = h
        self.precision = precision

    # -- error helper
    def _check(self, rc):
        if rc != 0:
            msg = C.create_string_buffer(1024)
            eb, wb = C.c_uint32(), C.c_uint32()
            self._lib.bhcb_last_error(self._h, msg, 1024, C.byref(eb), C.byref(wb))
            raise BhcbError(rc, msg.value.decode(errors="replace"), eb.value)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bhcb_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- bhc::setup
    def setup(self, file_root: str):
        self._check(self._lib.bhcb_setup(self._h, file_root.encode()))
        return self

    def add_env(self, file_root: str) -> int:
        idx = C.c_int32()
        self._check(self._lib.bhcb_add_env(self._h, file_root.encode(), C.byref(idx)))
        return idx.value

    def add_env_desc(self, desc) -> int:
        """Append an in-memory environment (an EnvDesc, or an EnvDescription)."""
        d = desc.desc if isinstance(desc, EnvDescription) else desc
        idx = C.c_int32()
        self._check(self._lib.bhcb_add_env_desc(self._h, C.byref(d), C.byref(idx)))
        return idx.value

    def ssp_at(self, env: int, r: float, z: float) -> float:
        """Sound speed (m/s) of environment env at range r and depth z (m)."""
        c = C.c_double()
        self._check(self._lib.bhcb_ssp_at(self._h, env, float(r), float(z), C.byref(c)))
        return c.value

    def clear(self):
        self._check(self._lib.bhcb_clear(self._h))

    def set_frequencies(self, env: int, freqs: Sequence[float]):
        arr = (C.c_double * len(freqs))(*[float(f) for f in freqs])
        self._check(self._lib.bhcb_set_frequencies(self._h, env, len(freqs), arr))

    # -- bhc::run
    def run(self):
        self._check(self._lib.bhcb_run(self._h))
        return self

    def prepare(self):
        self._check(self._lib.bhcb_prepare(self._h))

    def launch(self):
        self._check(self._lib.bhcb_launch(self._h))

    def sync(self):
        self._check(self._lib.bhcb_sync(self._h))

    # -- outputs
    def field_shape(self, env: int = 0):
        v = [C.c_int32() for _ in range(4)]
        self._check(self._lib.bhcb_field_shape(self._h, env, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def field(self, env: int = 0, ifreq: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Scaled complex pressure, shape (NSz, NRz_per_range, NRr), complex64."""
        _, nsz, nrz, nrr = self.field_shape(env)
        if out is None:
            out = np.empty((nsz, nrz, nrr), np.complex64)
        self._check(self._lib.bhcb_copy_field(self._h, env, ifreq, out.ctypes.data, out.nbytes))
        return out

    def field_device_ptr(self, env: int = 0, ifreq: int = 0) -> int:
        p = C.c_void_p()
        self._check(self._lib.bhcb_field_device(self._h, env, ifreq, C.byref(p)))
        return p.value

    def receivers(self, env: int = 0):
        _, _, _, nrr = self.field_shape(env)
        info_rz = self.field_shape(env)[2]
        rr = np.zeros(nrr, np.float64)
        rz = np.zeros(max(info_rz, 1), np.float32)
        self._check(self._lib.bhcb_receivers(self._h, env, rr.ctypes.data_as(C.POINTER(C.c_double)),
                                             nrr, rz.ctypes.data_as(C.POINTER(C.c_float)), rz.size))
        return rr, rz

    # -- 3-D (BELLHOP3D field modes)
    def setup3d(self, file_root: str):
        """bhc::setup<true, true>: FileRoot.env read as a 3-D run."""
        self._check(self._lib.bhcb_setup3d(self._h, file_root.encode()))
        return self

    def add_env3d(self, file_root: str) -> int:
        idx = C.c_int32()
        self._check(self._lib.bhcb_add_env3d(self._h, file_root.encode(), C.byref(idx)))
        return idx.value

    def field_shape3d(self, env: int = 0):
        """(NSz, NSx, NSy, Ntheta, NRz, NRr) of a 3-D environment's field."""
        dims = (C.c_int32 * 6)()
        self._check(self._lib.bhcb_field_shape3d(self._h, env, dims))
        return tuple(int(d) for d in dims)

    def field3d(self, env: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        """3-D pressure field, shape (NSz, NSx, NSy, Ntheta, NRz, NRr), complex64."""
        shape = self.field_shape3d(env)
        if out is None:
            out = np.empty(shape, np.complex64)
        self._check(self._lib.bhcb_copy_field(self._h, env, 0, out.ctypes.data, out.nbytes))
        return out

    def grid3d(self, env: int = 0) -> dict:
        """Source / receiver coordinates of a 3-D environment (m, m, m, m, m, deg)."""
        nsz, nsx, nsy, nth, nrz, nrr = self.field_shape3d(env)
        g = {"sx": np.zeros(nsx), "sy": np.zeros(nsy), "sz": np.zeros(nsz, np.float32),
             "rr": np.zeros(nrr), "rz": np.zeros(nrz, np.float32), "theta": np.zeros(nth)}
        self._check(self._lib.bhcb_grid3d(self._h, env, *[g[k].ctypes.data for k in
                                                            ("sx", "sy", "sz", "rr", "rz", "theta")]))
        return g

    def writeout(self, file_root: str, env: int = 0, ifreq: int = 0):
        self._check(self._lib.bhcb_writeout(self._h, env, ifreq, file_root.encode()))

    def set_arrival_options(self, max_narr: int = 0, allow_merging: bool = True):
        """ArrInfo::MaxNArr (0: sized from max_memory) and AllowMerging for arrivals runs."""
        self._check(self._lib.bhcb_set_arrival_options(self._h, int(max_narr), int(bool(allow_merging))))

    def arrivals(self, env: int = 0, ifreq: int = 0):
        """(narr [NSz, NRz_per_range, NRr] int32, arr [..., max_narr] ARRIVAL_DTYPE) of an arrivals run."""
        v = [C.c_int32() for _ in range(4)]
        self._check(self._lib.bhcb_arrivals_shape(self._h, env, ifreq, *[C.byref(x) for x in v]))
        nsz, nrzp, nrr, mx = (x.value for x in v)
        narr = np.zeros((nsz, nrzp, nrr), dtype=np.int32)
        arr = np.zeros((nsz, nrzp, nrr, mx), dtype=ARRIVAL_DTYPE)
        self._check(self._lib.bhcb_copy_arrivals(self._h, env, ifreq, narr.ctypes.data, narr.nbytes,
                                                 arr.ctypes.data, arr.nbytes))
        return narr, arr

    def eigen_hits(self, env: int = 0, ifreq: int = 0) -> np.ndarray:
        """Eigenray hits (EIGEN_HIT_DTYPE) of an eigen run, in the reference's order."""
        n = C.c_int64()
        self._check(self._lib.bhcb_eigen_hits(self._h, env, ifreq, None, 0, C.byref(n)))
        hits = np.zeros(n.value, dtype=EIGEN_HIT_DTYPE)
        if n.value:
            self._check(self._lib.bhcb_eigen_hits(self._h, env, ifreq, hits.ctypes.data, n.value, C.byref(n)))
        return hits

    def run_noalloc(self, field_dev_ptr: int, nbytes: int, env: int = 0, ifreq: int = 0):
        """Allocation-free run of one field into a caller-owned device buffer
        (see bhcb_run_noalloc in include/bhcb.h); the context must be prepared."""
        msg = C.create_string_buffer(256)
        rc = self._lib.bhcb_run_noalloc(self._h, env, ifreq, C.c_void_p(field_dev_ptr), nbytes, msg, 256)
        if rc != 0:
            raise BhcbError(rc, msg.value.decode(errors="replace"))

    def graph(self, field_dev_ptr: int, nbytes: int, env: int = 0, ifreq: int = 0) -> "FieldGraph":
        """Capture one field of the prepared context into a CUDA graph writing to field_dev_ptr."""
        g = C.c_void_p()
        msg = C.create_string_buffer(512)
        rc = self._lib.bhcb_graph_create(self._h, env, ifreq, C.c_void_p(field_dev_ptr), nbytes, C.byref(g),
                                         msg, len(msg))
        if rc != 0:
            raise BhcbError(rc, msg.value.decode(errors="replace"))
        return FieldGraph(self._lib, g)

    def rays(self, env: int = 0, ifreq: int = 0, dim: int = 2) -> List[dict]:
        """Ray trajectories of a ray run ('R') or the eigenrays of an eigen run
        ('E'): one dict per ray with alpha (deg), ntop, nbot and rz (n x 2,
        m; dim=3 for 3-D contexts: n x 3 points x, y, z)."""
        nr, npnt = C.c_int64(), C.c_int64()
        self._check(self._lib.bhcb_rays_shape(self._h, env, ifreq, C.byref(nr), C.byref(npnt)))
        n, m = nr.value, npnt.value
        npts = np.zeros(max(n, 1), np.int32)
        bnc = np.zeros(2 * max(n, 1), np.int32)
        alpha = np.zeros(max(n, 1))
        rz = np.zeros((max(m, 1), dim))
        self._check(self._lib.bhcb_copy_rays(self._h, env, ifreq, npts.ctypes.data, bnc.ctypes.data,
                                             alpha.ctypes.data, rz.ctypes.data, rz.nbytes))
        out, o = [], 0
        for i in range(n):
            out.append({"alpha": float(alpha[i]), "ntop": int(bnc[2 * i]), "nbot": int(bnc[2 * i + 1]),
                        "rz": rz[o:o + npts[i]].copy()})
            o += int(npts[i])
        return out

    def autotune(self, repeats: int = 2) -> dict:
        """Time the prepared TL workload with each launch shape; keep the fastest."""
        t = Tuning()
        self._check(self._lib.bhcb_autotune(self._h, repeats, C.byref(t)))
        return {"trace_block": t.trace_block, "influence_ctas_per_sm": t.influence_ctas_per_sm,
                "stage_kb": t.stage_kb, "trace_ms": t.trace_ms, "influence_ms": t.influence_ms,
                "trace_lanes": t.trace_lanes}

    def set_tuning(self, trace_block: int, influence_ctas_per_sm: int, stage_kb: int = 32, trace_lanes: int = 32):
        t = Tuning(trace_block, influence_ctas_per_sm, stage_kb, 0.0, 0.0, trace_lanes)
        self._check(self._lib.bhcb_set_tuning(self._h, C.byref(t)))

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        self._check(self._lib.bhcb_stream(self._h, C.byref(p)))
        return p.value or 0

    def stats(self) -> dict:
        s = Stats()
        self._check(self._lib.bhcb_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}


class FieldGraph:
    """A captured field run (bhcb_graph_*): launch() replays it, status() waits and checks."""

    def __init__(self, lib, handle):
        self._lib, self._g = lib, handle

    def launch(self, stream: int = 0):
        rc = self._lib.bhcb_graph_launch(self._g, C.c_void_p(stream or None))
        if rc != 0:
            raise BhcbError(rc, "graph launch failed")

    def status(self, stream: int = 0) -> dict:
        eb, ev = C.c_uint32(), C.c_uint64()
        rc = self._lib.bhcb_graph_status(self._g, C.c_void_p(stream or None), C.byref(eb), C.byref(ev))
        if rc not in (0, 4):
            raise BhcbError(rc, "graph status failed")
        return {"err_bits": eb.value, "evals": ev.value}

    def close(self):
        if self._g:
            self._lib.bhcb_graph_destroy(self._g)
            self._g = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def tl_db(p: np.ndarray) -> np.ndarray:
    """Transmission loss -20 log10 |p| (dB), +inf where p == 0."""
    a = np.abs(p).astype(np.float64)
    with np.errstate(divide="ignore"):
        return -20.0 * np.log10(a)
