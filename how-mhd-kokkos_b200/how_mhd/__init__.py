"""how_mhd -- Python mirror of the HOW-MHD driver-level interface over the C ABI
of libhowmhd.so (include/how_mhd.h).

The functions keep the reference's names and argument meaning
(jeongbhin/HOW-MHD-Kokkos: read_parameters, init_problem, bound,
bound_bfield, initialize_bfield_from_q, tstep, ssprk, prot, register_problem)
with a device-resident `Domain` in place of the Kokkos View `q` and the
module-global face-B arrays.  Errors raise `HowError` carrying the C status and
message; nothing aborts.  The CUDA library is required: importing this module
without libhowmhd.so raises ImportError (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIBPATH = Path(os.environ.get("HOW_MHD_LIB", _HERE.parent / "libhowmhd.so"))

HOW_OK = 0
HOW_BC_PERIODIC, HOW_BC_OPEN = 0, 1
HOW_PREC_FP64, HOW_PREC_MIXED = 0, 1
_ERRNAMES = {-1: "ARG", -2: "PARSE", -3: "PROBLEM", -4: "CUDA", -5: "NODEVICE",
             -6: "NONFINITE", -7: "DT", -8: "STATE"}


class HowError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"HOW_ERR_{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    """struct how_params (include/how_mhd.h), i.e. the reference's Parameters."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("nt", ctypes.c_int), ("nstep", ctypes.c_int), ("ntime", ctypes.c_int),
        ("xsize", ctypes.c_double), ("ysize", ctypes.c_double), ("zsize", ctypes.c_double),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("gam", ctypes.c_double), ("cour", ctypes.c_double), ("tend", ctypes.c_double),
        ("rhomin", ctypes.c_double), ("pgmin", ctypes.c_double),
        ("bc", ctypes.c_int * 3),
        ("px", ctypes.c_int), ("py", ctypes.c_int), ("pz", ctypes.c_int),
        ("problem", ctypes.c_char * 64),
        ("output_format", ctypes.c_char * 16),
        ("precision", ctypes.c_int),
        ("router", ctypes.c_int),
        ("seed", ctypes.c_uint64),
        ("problem_par", ctypes.c_double * 8),
        ("ct_avg", ctypes.c_int),
    ]

    @property
    def shape(self):
        return (self.nx + 6, self.ny + 6, self.nz + 6)


class PartInfo(ctypes.Structure):
    """struct how_part_info (include/how_mhd.h): one part's decomposition plan."""
    _fields_ = [(k, ctypes.c_int) for k in ("kstart", "nz", "z_sides", "lo_part", "hi_part", "nplanes",
                                            "send_up_first", "recv_lo_first", "send_down_first", "recv_hi_first")]


PROBLEM_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(Params), ctypes.c_void_p)


def _load():
    if not _LIBPATH.exists():
        raise ImportError(f"libhowmhd.so not found at {_LIBPATH}; build it with "
                          f"`make -C {_HERE.parent}` (CUDA sm_100a); there is no CPU fallback")
    lib = ctypes.CDLL(str(_LIBPATH))
    D = ctypes.POINTER(ctypes.c_double)
    P = ctypes.POINTER(Params)
    V = ctypes.c_void_p
    F = ctypes.POINTER(ctypes.c_float)
    U64P = ctypes.POINTER(ctypes.c_ulonglong)
    sig = {
        "how_params_default": ([P], ctypes.c_int),
        "how_parse_input": ([ctypes.c_char_p, P], ctypes.c_int),
        "how_parse_input_string": ([ctypes.c_char_p, P], ctypes.c_int),
        "how_finalize_params": ([P], ctypes.c_int),
        "how_register_problem": ([ctypes.c_char_p, PROBLEM_FN, V], ctypes.c_int),
        "how_list_problems": ([ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "how_problem_init_host": ([P, D], ctypes.c_int),
        "how_create": ([P, ctypes.POINTER(V)], ctypes.c_int),
        "how_destroy": ([V], ctypes.c_int),
        "how_last_error": ([], ctypes.c_char_p),
        "how_get_params": ([V, P], ctypes.c_int),
        "how_device_bytes": ([V], ctypes.c_size_t),
        "how_init_problem": ([V], ctypes.c_int),
        "how_set_state": ([V, ctypes.c_int, D], ctypes.c_int),
        "how_get_state": ([V, ctypes.c_int, D], ctypes.c_int),
        "how_set_face_b": ([V, ctypes.c_int, D, D, D], ctypes.c_int),
        "how_get_face_b": ([V, ctypes.c_int, D, D, D], ctypes.c_int),
        "how_bound": ([V, ctypes.c_int], ctypes.c_int),
        "how_bound_bfield": ([V, ctypes.c_int], ctypes.c_int),
        "how_init_bfield_from_q": ([V], ctypes.c_int),
        "how_tstep": ([V, D], ctypes.c_int),
        "how_ssprk": ([V, ctypes.c_double], ctypes.c_int),
        "how_prot": ([V, ctypes.c_int], ctypes.c_int),
        "how_sweep": ([V, ctypes.c_int, ctypes.c_double], ctypes.c_int),
        "how_fluxct": ([V, ctypes.c_int, ctypes.c_double, ctypes.c_double], ctypes.c_int),
        "how_set_wait_limit": ([V, ctypes.c_int], ctypes.c_int),
        "how_get_ct_array": ([V, ctypes.c_int, D], ctypes.c_int),
        "how_run": ([V, D, ctypes.c_long, ctypes.POINTER(ctypes.c_long), D, ctypes.c_long], ctypes.c_int),
        "how_output": ([V, ctypes.c_int, ctypes.c_double, ctypes.c_char_p], ctypes.c_int),
        "how_output_async": ([V, ctypes.c_int, ctypes.c_double, ctypes.c_char_p], ctypes.c_int),
        "how_output_wait": ([V], ctypes.c_int),
        "how_set_precision": ([V, ctypes.c_int], ctypes.c_int),
        "how_sync": ([V], ctypes.c_int),
        "how_kernel_launches": ([V], ctypes.c_long),
        "how_stream": ([V], ctypes.c_void_p),
        "how_set_kernel_timing": ([V, ctypes.c_int], ctypes.c_int),
        "how_get_kernel_timing": ([V, D, ctypes.POINTER(ctypes.c_long)], ctypes.c_int),
        "how_measure_fp64_peak": ([D, ctypes.c_int], ctypes.c_int),
        "how_sweep_phase_profile": ([V, ctypes.c_int, ctypes.c_double, D, ctypes.c_int], ctypes.c_int),
        "how_ensemble_create": ([P, ctypes.c_int, ctypes.POINTER(V)], ctypes.c_int),
        "how_ensemble_destroy": ([V], ctypes.c_int),
        "how_ensemble_size": ([V], ctypes.c_int),
        "how_ensemble_member": ([V, ctypes.c_int], V),
        "how_ensemble_init": ([V], ctypes.c_int),
        "how_ensemble_set_shapes": ([V, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "how_ensemble_get_shapes": ([V, ctypes.POINTER(ctypes.c_int), D], ctypes.c_int),
        "how_ensemble_shape_info": ([ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "how_ensemble_run": ([V, ctypes.c_long, ctypes.POINTER(ctypes.c_long)], ctypes.c_int),
        "how_ensemble_member_status": ([V, ctypes.c_int, D, ctypes.POINTER(ctypes.c_long),
                                        ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "how_ensemble_graph_launches": ([V], ctypes.c_long),
        "how_ensemble_stream": ([V], ctypes.c_void_p),
        "how_part_plan": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(PartInfo)],
                          ctypes.c_int),
        "how_group_create": ([P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(V)], ctypes.c_int),
        "how_group_destroy": ([V], ctypes.c_int),
        "how_group_size": ([V], ctypes.c_int),
        "how_group_part": ([V, ctypes.c_int], V),
        "how_group_part_range": ([V, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
                                 ctypes.c_int),
        "how_group_init": ([V], ctypes.c_int),
        "how_group_set_state": ([V, D], ctypes.c_int),
        "how_group_run": ([V, D, ctypes.c_long, ctypes.POINTER(ctypes.c_long), D, ctypes.c_long], ctypes.c_int),
        "how_group_get_state": ([V, D], ctypes.c_int),
        "how_group_get_face_b": ([V, D, D, D], ctypes.c_int),
        "how_group_output": ([V, ctypes.c_int, ctypes.c_double, ctypes.c_char_p], ctypes.c_int),
        "how_router_param_count": ([], ctypes.c_int),
        "how_router_default": ([F, ctypes.c_int, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
        "how_router_set_weights": ([V, F, ctypes.c_int], ctypes.c_int),
        "how_router_configure": ([V, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float], ctypes.c_int),
        "how_router_stats": ([V, U64P, U64P, ctypes.c_int], ctypes.c_int),
        "how_router_set_refresh": ([V, ctypes.c_int], ctypes.c_int),
        "how_router_stats4": ([V, U64P, U64P, U64P, U64P, ctypes.c_int], ctypes.c_int),
        "how_collect_begin": ([V, ctypes.c_uint, ctypes.c_uint], ctypes.c_int),
        "how_collect_end": ([V, F, ctypes.c_uint, ctypes.POINTER(ctypes.c_uint)], ctypes.c_int),
        "how_router_train": ([F, F, F, ctypes.c_long, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                              ctypes.c_ulonglong, F], ctypes.c_int),
        "how_router_grad": ([F, F, F, ctypes.c_long, ctypes.c_float, F, F], ctypes.c_int),
        "how_router_infer": ([F, F, ctypes.c_long, F, F], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


_lib = _load()
LIBRARY_PATH = str(_LIBPATH)


def _check(rc):
    if rc != HOW_OK:
        raise HowError(rc, _lib.how_last_error().decode(errors="replace"))


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f32(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def lib():
    """The loaded ctypes library (for instrumentation)."""
    return _lib


# --------------------------------------------------------------- parameters
def default_parameters() -> Params:
    p = Params()
    _check(_lib.how_params_default(ctypes.byref(p)))
    return p


def read_parameters(source) -> Params:
    """read_parameters + finalize_parameters_after_read (src/parameters.cpp:7-160).

    `source` is a path to an input.in file or the text itself (contains a newline)."""
    p = Params()
    if isinstance(source, (str, os.PathLike)) and "\n" not in str(source) and Path(source).exists():
        _check(_lib.how_parse_input(str(source).encode(), ctypes.byref(p)))
    else:
        _check(_lib.how_parse_input_string(str(source).encode(), ctypes.byref(p)))
    return p


def make_parameters(**kw) -> Params:
    """Parameters from keywords using the input.in key names (bc as strings)."""
    lines = []
    for k, v in kw.items():
        # repr of a float round-trips exactly (numpy scalars as plain floats)
        lines.append(f"{k} {float(v)!r}" if isinstance(v, float) else f"{k} {v}")
    return read_parameters("\n".join(lines) + "\n")


# ------------------------------------------------------------------ problems
_registered_callbacks = []


def register_problem(name: str, fn) -> None:
    """register_problem (src/problem.hpp:8-22).  fn(q, params) fills one stage of q
    (numpy array (8, nx+6, ny+6, nz+6), reference layout) in place."""
    def cb(qptr, pptr, user):
        try:
            p = pptr.contents
            q = np.ctypeslib.as_array(qptr, shape=(8,) + p.shape)
            fn(q, p)
            return 0
        except Exception:   # noqa: BLE001 -- reported as a C status
            return 1
    c = PROBLEM_FN(cb)
    _registered_callbacks.append(c)
    _check(_lib.how_register_problem(name.encode(), c, None))


def list_problems():
    buf = ctypes.create_string_buffer(1 << 14)
    _lib.how_list_problems(buf, len(buf))
    return [s for s in buf.value.decode().split("\n") if s]


def problem_state(params: Params) -> np.ndarray:
    """init_problem on the host: stage 0 of q in the reference layout."""
    q = np.zeros((8,) + params.shape)
    _check(_lib.how_problem_init_host(ctypes.byref(params), _dptr(q)))
    return q


# -------------------------------------------------------------------- domain
class Domain:
    """Device-resident q(6 stages) + face B + CT arrays of one run (how_ctx)."""

    def __init__(self, params: Params):
        self.params = params
        h = ctypes.c_void_p()
        _check(_lib.how_create(ctypes.byref(params), ctypes.byref(h)))
        self._h = h
        p = Params()
        _check(_lib.how_get_params(h, ctypes.byref(p)))
        self.params = p
        self.shape = p.shape

    @classmethod
    def _borrowed(cls, handle, owner, part=None):
        """A view of a context owned by someone else (an ensemble member, or
        part `part` of a decomposed group)."""
        d = cls.__new__(cls)
        d._h = ctypes.c_void_p(handle)
        d._owner = owner
        d._part = part
        p = Params()
        _check(_lib.how_get_params(d._h, ctypes.byref(p)))
        d.params = p
        d.shape = p.shape
        return d

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.how_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # state
    def set_state(self, q, stage=0):
        q = np.ascontiguousarray(q, dtype=np.float64)
        if q.shape != (8,) + self.shape:
            raise ValueError(f"state shape {q.shape} != {(8,) + self.shape}")
        _check(_lib.how_set_state(self._h, stage, _dptr(q)))

    def get_state(self, stage=0, out=None):
        q = out if out is not None else np.empty((8,) + self.shape)
        _check(_lib.how_get_state(self._h, stage, _dptr(q)))
        return q

    def set_face_b(self, bx, by, bz, stage=0):
        arrs = [np.ascontiguousarray(b, dtype=np.float64) for b in (bx, by, bz)]
        _check(_lib.how_set_face_b(self._h, stage, *(_dptr(a) for a in arrs)))

    def get_face_b(self, stage=0):
        b = [np.empty(self.shape) for _ in range(3)]
        _check(_lib.how_get_face_b(self._h, stage, *(_dptr(x) for x in b)))
        return b

    def get_face_b_into(self, bx, by, bz, stage=0):
        for x in (bx, by, bz):
            if x.shape != self.shape or x.dtype != np.float64 or not x.flags.c_contiguous:
                raise ValueError("face-B buffers must be C-contiguous float64 of the padded shape")
        _check(_lib.how_get_face_b(self._h, stage, _dptr(bx), _dptr(by), _dptr(bz)))

    def get_ct_array(self, which):
        a = np.empty(self.shape)
        _check(_lib.how_get_ct_array(self._h, which, _dptr(a)))
        return a

    # path functions
    def init_problem(self):
        _check(_lib.how_init_problem(self._h))

    def bound(self, stage):
        _check(_lib.how_bound(self._h, stage))

    def bound_bfield(self, stage):
        _check(_lib.how_bound_bfield(self._h, stage))

    def initialize_bfield_from_q(self):
        _check(_lib.how_init_bfield_from_q(self._h))

    def tstep(self) -> float:
        dt = ctypes.c_double()
        _check(_lib.how_tstep(self._h, ctypes.byref(dt)))
        return dt.value

    def ssprk(self, dt: float):
        _check(_lib.how_ssprk(self._h, dt))

    def prot(self, stage):
        _check(_lib.how_prot(self._h, stage))

    def sweep(self, direction: int, dt: float):
        _check(_lib.how_sweep(self._h, direction, dt))

    def fluxct(self, iw: int, k1: float, k3: float):
        """fluxct(q, iw, k1, k3, par, ct) (src/fluxct.cpp:786-899) on the CT
        flux arrays the last sweeps filled, after bound_bfield(iw - 1)."""
        _check(_lib.how_fluxct(self._h, iw, k1, k3))

    def set_wait_limit(self, expire_at_once: bool):
        """Failure-detection tests: make the sweep kernels' tile waits give up at once."""
        _check(_lib.how_set_wait_limit(self._h, 1 if expire_at_once else 0))

    def run(self, time=0.0, max_steps=-1, dts_cap=0):
        t = ctypes.c_double(time)
        s = ctypes.c_long(0)
        dts = np.zeros(max(dts_cap, 1))
        _check(_lib.how_run(self._h, ctypes.byref(t), max_steps, ctypes.byref(s), _dptr(dts), dts_cap))
        return t.value, s.value, dts[: min(s.value, dts_cap)].copy()

    def _dump_path(self, step, d):
        fmt = self.params.output_format.decode() if isinstance(self.params.output_format, bytes) \
            else str(self.params.output_format)
        if fmt == "none":
            return None
        rank = "" if getattr(self, "_part", None) is None else "_rank%06d" % self._part
        name = "dump%06d%s%s" % (int(step), rank, ".dat" if fmt == "dat" else ".vts")
        return name if d == "" else d + "/" + name

    def output(self, step, time, directory=None):
        """Write the dump file of q(0) in the parameters' output_format, as
        the reference's output(q, par, step, time) (src/output.cpp:555-572):
        <directory>/dumpNNNNNN.dat or .vts, directory "output" by default.
        Returns the file's path (None for output_format none)."""
        d = "output" if directory is None else str(directory)
        _check(_lib.how_output(self._h, int(step), float(time), d.encode()))
        return self._dump_path(step, d)

    def output_async(self, step, time, directory=None):
        """The same dump, written while later steps run; output_wait() joins."""
        d = "output" if directory is None else str(directory)
        _check(_lib.how_output_async(self._h, int(step), float(time), d.encode()))
        return self._dump_path(step, d)

    def output_wait(self):
        _check(_lib.how_output_wait(self._h))

    def sweep_phase_profile(self, direction: int, dt: float):
        """Mean cycles per block of each sweep phase (instrumentation)."""
        out = np.zeros(12)
        _check(_lib.how_sweep_phase_profile(self._h, direction, dt, _dptr(out), 12))
        return out

    def set_precision(self, mode):
        if isinstance(mode, str):
            mode = {"fp64": HOW_PREC_FP64, "mixed": HOW_PREC_MIXED}[mode]
        _check(_lib.how_set_precision(self._h, mode))

    def sync(self):
        _check(_lib.how_sync(self._h))

    # ---- learned routing
    def set_router(self, weights, mode="learned", threshold=0.0, guard_jump=0.25, guard_floor=100.0):
        """Route interfaces between full characteristic WENO5 and the linear
        flux.  mode: "off", "learned" (network + guard) or "guard" (guard only)."""
        m = {"off": 0, "learned": 1, "guard": 2}[mode] if isinstance(mode, str) else int(mode)
        if weights is not None:
            w = _f32(weights, ROUTER_PARAMS)
            _check(_lib.how_router_set_weights(self._h, _fptr(w), w.size))
        _check(_lib.how_router_configure(self._h, m, threshold, guard_jump, guard_floor))

    def set_router_refresh(self, stages):
        """Learned routing: the network's decisions every `stages` SSPRK
        stages of a step (5 = once per step, the default; 1 = every stage), or
        with 10 once every second step; the guard is evaluated at every
        stage."""
        _check(_lib.how_router_set_refresh(self._h, int(stages)))

    def router_stats(self, reset=False, groups=False):
        """(full, cheap) interface counts since the last reset; with groups=True
        also the 16-interface groups inferred on the tensor cores and the flat
        groups that used the precomputed logit."""
        v = [ctypes.c_ulonglong(0) for _ in range(4)]
        _check(_lib.how_router_stats4(self._h, *(ctypes.byref(x) for x in v), int(reset)))
        return tuple(x.value for x in v) if groups else (v[0].value, v[1].value)

    def collect_begin(self, capacity, every=1):
        _check(_lib.how_collect_begin(self._h, capacity, every))
        self._collect_cap = capacity

    def collect_end(self):
        """Records (n, 8): 6 features, the largest departure of the nonlinear
        WENO weights from the linear ones, and the flux departure (what the
        cheap flux would change: dt/dx |F_full - F_linear| over the local size
        of the conserved variable, largest component)."""
        cap = getattr(self, "_collect_cap", 0)
        out = np.zeros((max(cap, 1), 8), np.float32)
        n = ctypes.c_uint(0)
        _check(_lib.how_collect_end(self._h, _fptr(out), cap, ctypes.byref(n)))
        return out[: n.value].copy()

    @property
    def kernel_launches(self) -> int:
        return _lib.how_kernel_launches(self._h)

    @property
    def stream(self) -> int:
        return _lib.how_stream(self._h) or 0

    @property
    def device_bytes(self) -> int:
        return _lib.how_device_bytes(self._h)


# ---------------------------------------------------------------- ensembles
def part_plan(nz, nparts, periodic_z, part) -> PartInfo:
    """The decomposition plan of one part (how_part_plan; host only)."""
    r = PartInfo()
    _check(_lib.how_part_plan(nz, nparts, 1 if periodic_z else 0, part, ctypes.byref(r)))
    return r


class Group:
    """A domain decomposed into z slabs (how_group): one context per part,
    each on its own stream (and, with `devices`, its own GPU), stepped
    together; the halos move as copies of whole z planes between the parts.
    The decomposed run equals the whole-domain run bit for bit."""

    def __init__(self, params, nparts, devices=None):
        h = ctypes.c_void_p()
        dev = None if devices is None else (ctypes.c_int * nparts)(*devices)
        _check(_lib.how_group_create(ctypes.byref(params), nparts, dev, ctypes.byref(h)))
        self._h = h
        self.params = params
        self.n = nparts
        self.shape = params.shape
        self.parts = [Domain._borrowed(_lib.how_group_part(h, k), self, part=k) for k in range(nparts)]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            for d in self.parts:
                d._h = None
            _lib.how_group_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def part_range(self, k):
        """(first global active z plane, number of planes) of part k."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(_lib.how_group_part_range(self._h, k, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def init_problem(self):
        _check(_lib.how_group_init(self._h))

    def set_state(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        if q.shape != (8,) + self.shape:
            raise ValueError(f"state shape {q.shape} != {(8,) + self.shape}")
        _check(_lib.how_group_set_state(self._h, _dptr(q)))

    def run(self, time=0.0, max_steps=-1, dts_cap=0):
        t = ctypes.c_double(time)
        s = ctypes.c_long(0)
        dts = np.zeros(max(dts_cap, 1))
        _check(_lib.how_group_run(self._h, ctypes.byref(t), max_steps, ctypes.byref(s), _dptr(dts), dts_cap))
        return t.value, s.value, dts[: min(s.value, dts_cap)].copy()

    def get_state(self):
        """Active cells of stage 0 in a global reference-layout array (ghosts zero)."""
        q = np.zeros((8,) + self.shape)
        _check(_lib.how_group_get_state(self._h, _dptr(q)))
        return q

    def get_face_b(self):
        b = [np.zeros(self.shape) for _ in range(3)]
        _check(_lib.how_group_get_face_b(self._h, *(_dptr(x) for x in b)))
        return b

    def output(self, step, time, directory=None):
        """Every part's dump piece, as the reference's MPI rank of the same
        slab writes it (<directory>/dumpNNNNNN_rankPPPPPP.dat or .vts), and for
        .vts the PStructuredGrid master <directory>/dumpNNNNNN.pvts.  Returns
        (master path or None, [piece paths]); (None, []) for output_format none."""
        d = "output" if directory is None else str(directory)
        _check(_lib.how_group_output(self._h, int(step), float(time), d.encode()))
        pieces = [p._dump_path(step, d) for p in self.parts]
        if pieces[0] is None:
            return None, []
        master = None
        if pieces[0].endswith(".vts"):
            name = "dump%06d.pvts" % int(step)
            master = name if d == "" else d + "/" + name
        return master, pieces


class Ensemble:
    """A batched ensemble (how_ensemble): independent runs of uneven sizes
    advanced together, one launch per kernel for all members, one CUDA graph
    per step."""

    def __init__(self, params_list):
        arr = (Params * len(params_list))(*params_list)
        h = ctypes.c_void_p()
        _check(_lib.how_ensemble_create(arr, len(params_list), ctypes.byref(h)))
        self._h = h
        self.n = len(params_list)
        self.members = [Domain._borrowed(_lib.how_ensemble_member(h, m), self) for m in range(self.n)]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            for d in self.members:
                d._h = None
            _lib.how_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init(self):
        _check(_lib.how_ensemble_init(self._h))

    @property
    def stream(self):
        """The ensemble's CUDA stream handle (cudaStream_t as an int)."""
        return _lib.how_ensemble_stream(self._h)

    def set_shapes(self, sx, sy, sz=0):
        _check(_lib.how_ensemble_set_shapes(self._h, sx, sy, sz))

    def shapes(self):
        """(chosen shape per direction, autotuner sweep ms [dir][candidate])"""
        s = (ctypes.c_int * 3)()
        ms = np.zeros(9)
        _check(_lib.how_ensemble_get_shapes(self._h, s, _dptr(ms)))
        return list(s), ms.reshape(3, 3)

    @staticmethod
    def shape_info(direction, shape):
        a, b = ctypes.c_int(0), ctypes.c_int(0)
        _check(_lib.how_ensemble_shape_info(direction, shape, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def run(self, max_steps=-1):
        s = ctypes.c_long(0)
        _check(_lib.how_ensemble_run(self._h, max_steps, ctypes.byref(s)))
        return s.value

    def status(self, m):
        """(time, steps, done) of member m"""
        t, s, d = ctypes.c_double(0), ctypes.c_long(0), ctypes.c_int(0)
        _check(_lib.how_ensemble_member_status(self._h, m, ctypes.byref(t), ctypes.byref(s), ctypes.byref(d)))
        return t.value, s.value, bool(d.value)

    @property
    def graph_launches(self):
        return _lib.how_ensemble_graph_launches(self._h)


# ------------------------------------------------------------ router training
ROUTER_PARAMS = _lib.how_router_param_count()


def default_router():
    """(weights, logit threshold) built into the library (`router on`)."""
    w = np.zeros(ROUTER_PARAMS, np.float32)
    t = ctypes.c_float(0)
    _check(_lib.how_router_default(_fptr(w), ROUTER_PARAMS, ctypes.byref(t)))
    return w, float(t.value)


def router_grad(w, feats, labels, pos_weight=1.0):
    """GPU gradient (and loss) of the mean weighted BCE at w."""
    w = _f32(w, ROUTER_PARAMS)
    x = _f32(feats)
    y = _f32(labels)
    g = np.zeros(ROUTER_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    _check(_lib.how_router_grad(_fptr(w), _fptr(x), _fptr(y), y.size, pos_weight, _fptr(g), _fptr(loss)))
    return g, float(loss[0])


def router_train(w, feats, labels, iters, batch=4096, lr=3e-3, pos_weight=1.0, seed=1):
    """Adam on the GPU; returns (weights, per-iteration loss)."""
    w = _f32(w, ROUTER_PARAMS).copy()
    x = _f32(feats)
    y = _f32(labels)
    hist = np.zeros(iters, np.float32)
    _check(_lib.how_router_train(_fptr(w), _fptr(x), _fptr(y), y.size, pos_weight, iters, batch, lr, seed,
                                 _fptr(hist)))
    return w, hist


def router_infer(w, feats):
    """(FP32 logits, BF16 tensor-core logits) of feature rows."""
    w = _f32(w, ROUTER_PARAMS)
    x = _f32(feats)
    n = x.size // 6
    a = np.zeros(n, np.float32)
    b = np.zeros(n, np.float32)
    _check(_lib.how_router_infer(_fptr(w), _fptr(x), n, _fptr(a), _fptr(b)))
    return a, b


# reference-named free functions over a Domain
def init_problem(dom: Domain):
    """init_problem + bound(q,0) + initialize_bfield_from_q (src/main.cpp:125-130)."""
    dom.init_problem()


def bound(dom: Domain, stage: int):
    dom.bound(stage)


def bound_bfield(dom: Domain, stage: int):
    dom.bound_bfield(stage)


def tstep(dom: Domain) -> float:
    return dom.tstep()


def ssprk(dom: Domain, dt: float):
    dom.ssprk(dt)


def prot(dom: Domain, stage: int):
    dom.prot(stage)


def fluxct(dom: Domain, iw: int, k1: float, k3: float):
    dom.fluxct(iw, k1, k3)
