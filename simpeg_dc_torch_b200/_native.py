"""ctypes binding of libdct (include/dct.h).

The shared library is built in-tree (`python -m simpeg_dc_torch_b200.build_lib`)
into `simpeg_dc_torch_b200/lib/libdct.so`.  Loading it needs no GPU; creating a
plan does.  There is no fallback: a missing library raises at first use.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# DCT_LIB_PATH selects another build of the same sources (for example one
# compiled with different -D knobs, to compare kernels); unset: the in-tree build
LIB_PATH = os.environ.get("DCT_LIB_PATH") or os.path.join(_HERE, "lib", "libdct.so")

F64, F32, C128 = 0, 1, 2

STATUS = {
    0: "OK", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
    4: "non-positive pivot (matrix not SPD)",
    5: "iterative refinement did not converge", 6: "pattern rejected",
    7: "solve before factorize", 8: "no CUDA device",
    9: "a bounded device wait timed out",
}


class DCTError(RuntimeError):
    """A libdct entry point returned a non-zero status."""

    def __init__(self, code, where, msg):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, 'error')} "
                         f"(status {code}) {msg}".rstrip())


_lib = None
_lock = threading.Lock()

_p = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)


class SymbolicInfo(C.Structure):
    _fields_ = [("n", _i64), ("nnz_in", _i64), ("nsuper", _i64),
                ("nlevels", _i64), ("max_front", _i64), ("max_ns", _i64),
                ("nnz_L", _i64), ("front_total", _i64),
                ("flops_factor", C.c_double)]


class Tuning(C.Structure):
    """dct_tuning: the schedule shapes of a plan (0 = default)."""
    _fields_ = [("small_front_max", _i32), ("update_block", _i32),
                ("solve_target", _i32), ("solve_split_max", _i32),
                ("solve_split_min", _i32), ("small_tc", _i32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


_SIGS = {
    "dct_version": (C.c_int, []),
    "dct_last_error": (C.c_char_p, []),
    "dct_symbolic_create": (C.c_int, [_i32, _p, _p, _p, _i32, _i32,
                                      C.POINTER(_p)]),
    "dct_symbolic_destroy": (None, [_p]),
    "dct_symbolic_get_info": (C.c_int, [_p, C.POINTER(SymbolicInfo)]),
    "dct_symbolic_get_array": (C.c_int, [_p, C.c_char_p, _p, _i64, _pi64]),
    "dct_symbolic_get_schedule": (C.c_int, [_p, _i32, _i32, _p, _pi64, _p,
                                            _pi64]),
    "dct_plan_create": (C.c_int, [_p, _i32, _i32, _i32, _i32, C.POINTER(_p)]),
    "dct_selftest_wait_timeout": (C.c_int, [_i32, _pi32, _pi32, _p]),
    "dct_plan_create_general": (C.c_int, [_p, _i32, _i32, _i32, C.POINTER(_p)]),
    "dct_solve_transposed": (C.c_int, [_p, _p, _i32, _i32, _i32, _p, _p]),
    "dct_plan_static_pivots": (C.c_int, [_p, _p, _pi32]),
    "dct_plan_create_tuned": (C.c_int, [_p, _i32, _i32, _i32, _i32,
                                        C.POINTER(Tuning), C.POINTER(_p)]),
    "dct_tuning_default": (C.c_int, [_i32, C.POINTER(Tuning)]),
    "dct_plan_get_tuning": (C.c_int, [_p, C.POINTER(Tuning)]),
    "dct_plan_destroy": (None, [_p]),
    "dct_plan_set_refinement": (C.c_int, [_p, _i32]),
    "dct_plan_set_refinement_tolerance": (C.c_int, [_p, C.c_double]),
    "dct_plan_refinement_info": (C.c_int, [_p, _p, _pi32, _pi32,
                                           C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), _i32]),
    "dct_plan_iperm": (C.c_int, [_p, C.POINTER(_p)]),
    "dct_plan_stamp": (_i64, [_p]),
    "dct_factorize": (C.c_int, [_p, _p, _i32, _i64, _p]),
    "dct_solve": (C.c_int, [_p, _p, _i32, _i32, _i32, _p, _p]),
    "dct_solve_permuted": (C.c_int, [_p, _p, _i32, _i32, _p, _p]),
    "dct_plan_profile": (C.c_int, [_p, _i32, _i32]),
    "dct_plan_profile_get": (C.c_int, [_p, _i32, C.POINTER(C.c_double), _pi64,
                                       C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]),
    "dct_plan_profile_log": (C.c_int, [_p, _i64, _pi32, C.POINTER(C.c_double),
                                       _pi64]),
    "dct_check_status": (C.c_int, [_p, _p, _pi32, _pi32,
                                   C.POINTER(C.c_double)]),
    "dct_sigma_values": (C.c_int, [_i64, _p, _p, _p, _i64, _p, _p, _p, _p]),
    "dct_values_vjp": (C.c_int, [_i64, _p, _p, _p, _p, _p, _p, _p]),
    "dct_scatter_rhs": (C.c_int, [_i64, _i32, _i64, _p, _p, _p, _p, _p, _p,
                                  _p, _p]),
    "dct_project_data": (C.c_int, [_i32, _i64, _i32, _i64, _p, _p, _p, _p,
                                   _p, _p, _p, _p, _p]),
    "dct_gather_contract": (C.c_int, [_i32, _i64, _i64, _i32, _p, _p, _p, _p,
                                      _p, _p, _p, _p]),
    "dct_gather_contract_plain": (C.c_int, [_i32, _i64, _i64, _i32, _p, _p,
                                            _i32, _p, _p, _p, _p]),
    "dct_solve_small_noalloc": (C.c_int, [_i32, _p, _p, _p, _p, _i32, _p, _p]),
    "dct_csr_spmv": (C.c_int, [_i64, _p, _p, _p, _p, _p, _p]),
    "dct_pattern_spmm": (C.c_int, [_i32, _i32, _i32, _p, _p, _p, _p, _i64,
                                   C.c_double, _p, _p, _p]),
    "dct_gather_pairwise": (C.c_int, [_i32, _i64, _i64, _i32, _i32, _p, _p, _p,
                                      _p, _p, _p, _p, _p, _p]),
    "dct_values_vjp_multi": (C.c_int, [_i64, _i32, _p, _p, _p, _p, _p, _p, _p]),
}


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        f"libdct is not built ({LIB_PATH} missing); run "
                        "`python -m simpeg_dc_torch_b200.build_lib`")
                L = C.CDLL(LIB_PATH)
                for name, (res, args) in _SIGS.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def check(rc, where):
    if rc != 0:
        msg = lib().dct_last_error()
        raise DCTError(rc, where, msg.decode() if msg else "")


def exported_symbols():
    return list(_SIGS)


def _ptr(a):
    return a.ctypes.data_as(_p) if a is not None else None


class Symbolic:
    """Nested-dissection analysis of a CSR pattern (host only)."""

    _ARR64 = {"front_off", "rows_ptr", "rel_ptr", "amap_ptr"}

    def __init__(self, crow, col, coords=None, leaf_size=64):
        crow = np.ascontiguousarray(np.asarray(crow, dtype=np.int32))
        col = np.ascontiguousarray(np.asarray(col, dtype=np.int32))
        n = crow.size - 1
        ndim = 0
        if coords is not None:
            coords = np.ascontiguousarray(np.asarray(coords, dtype=np.int32))
            ndim = coords.shape[1]
        h = _p()
        check(lib().dct_symbolic_create(n, _ptr(crow), _ptr(col), _ptr(coords),
                                        ndim, int(leaf_size), C.byref(h)),
              "dct_symbolic_create")
        self._h = h
        self.n = n
        self.nnz = col.size

    @property
    def handle(self):
        return self._h

    def info(self):
        s = SymbolicInfo()
        check(lib().dct_symbolic_get_info(self._h, C.byref(s)),
              "dct_symbolic_get_info")
        return {k: getattr(s, k) for k, _ in SymbolicInfo._fields_}

    def array(self, name):
        size = C.c_int64(0)
        check(lib().dct_symbolic_get_array(self._h, name.encode(), None, 0,
                                           C.byref(size)), "get_array")
        dt = np.int64 if name in self._ARR64 else np.int32
        out = np.empty(size.value // np.dtype(dt).itemsize, dtype=dt)
        check(lib().dct_symbolic_get_array(self._h, name.encode(), _ptr(out),
                                           size.value, C.byref(size)),
              "get_array")
        return out

    def schedule(self, dtype, which):
        nt, nl = C.c_int64(0), C.c_int64(0)
        check(lib().dct_symbolic_get_schedule(self._h, dtype, which, None,
                                              C.byref(nt), None, C.byref(nl)),
              "get_schedule")
        tasks = np.empty((nt.value, 4), dtype=np.int32)
        launches = np.empty((nl.value, 5), dtype=np.int64)
        check(lib().dct_symbolic_get_schedule(self._h, dtype, which,
                                              _ptr(tasks), C.byref(nt),
                                              _ptr(launches), C.byref(nl)),
              "get_schedule")
        return tasks, launches

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.dct_symbolic_destroy(h)
            self._h = None


class Plan:
    """Numeric plan: nbatch systems on the pattern of `sym`, on one device."""

    def __init__(self, sym: Symbolic, nbatch, max_rhs, dtype, device, tuning=None,
                 general=False):
        h = _p()
        tu = None
        if tuning is not None:
            tu = Tuning(**{k: int(v) for k, v in dict(tuning).items()})
        if general:
            # float64 L U with static pivoting (unsymmetric values)
            check(lib().dct_plan_create_general(sym.handle, int(nbatch), int(max_rhs),
                                                int(device), C.byref(h)),
                  "dct_plan_create_general")
        else:
            check(lib().dct_plan_create_tuned(sym.handle, int(nbatch), int(max_rhs),
                                              int(dtype), int(device),
                                              None if tu is None else C.byref(tu),
                                              C.byref(h)),
                  "dct_plan_create_tuned")
        self.general = bool(general)
        self._h = h
        self.sym = sym
        self.nbatch, self.max_rhs, self.dtype = int(nbatch), int(max_rhs), dtype
        self.device = int(device)
        ip = _p()
        check(lib().dct_plan_iperm(h, C.byref(ip)), "dct_plan_iperm")
        self.d_iperm = ip.value

    @property
    def handle(self):
        return self._h

    def tuning(self):
        """The schedule shapes this plan was built with."""
        t = Tuning()
        check(lib().dct_plan_get_tuning(self._h, C.byref(t)), "dct_plan_get_tuning")
        return t.as_dict()

    def set_refinement(self, iters):
        check(lib().dct_plan_set_refinement(self._h, int(iters)),
              "dct_plan_set_refinement")

    def set_refinement_tolerance(self, tol):
        check(lib().dct_plan_set_refinement_tolerance(self._h, float(tol)),
              "dct_plan_set_refinement_tolerance")

    def refinement_info(self, stream):
        """(corrections, converged, estimated error, [rho_1 ..]) of the last
        float32 solve (synchronises the stream)."""
        it, conv = C.c_int32(0), C.c_int32(0)
        est = C.c_double(0.0)
        rho = (C.c_double * 16)()
        check(lib().dct_plan_refinement_info(self._h, stream, C.byref(it),
                                             C.byref(conv), C.byref(est), rho, 16),
              "dct_plan_refinement_info")
        return it.value, bool(conv.value), est.value, list(rho[:min(it.value, 16)])

    def stamp(self):
        return int(lib().dct_plan_stamp(self._h))

    def factorize(self, d_vals, vals_dtype, vals_stride, stream):
        check(lib().dct_factorize(self._h, d_vals, vals_dtype, int(vals_stride),
                                  stream), "dct_factorize")

    def solve(self, d_b, io_dtype, b_batched, k, d_x, stream):
        check(lib().dct_solve(self._h, d_b, io_dtype, int(b_batched), int(k),
                              d_x, stream), "dct_solve")

    def solve_transposed(self, d_b, io_dtype, b_batched, k, d_x, stream):
        check(lib().dct_solve_transposed(self._h, d_b, io_dtype, int(b_batched), int(k),
                                         d_x, stream), "dct_solve_transposed")

    def static_pivots(self, stream):
        n = C.c_int32(0)
        check(lib().dct_plan_static_pivots(self._h, stream, C.byref(n)),
              "dct_plan_static_pivots")
        return n.value

    def solve_permuted(self, d_bp, b_batched, k, d_xp, stream):
        check(lib().dct_solve_permuted(self._h, d_bp, int(b_batched), int(k),
                                       d_xp, stream), "dct_solve_permuted")

    KINDS = ("small_front", "large_scatter", "extend_add", "panel_trsm",
             "trailing_update", "panel_inverse", "linv_init", "linv_t",
             "linv_x", "fwd_small", "fwd_linv", "fwd_bnd", "bwd_small",
             "bwd_gemm", "bwd_linv", "fwd_linv_tc", "fwd_bnd_tc",
             "bwd_gemm_tc", "bwd_linv_tc")

    def profile(self, enable, reset=True):
        check(lib().dct_plan_profile(self._h, int(bool(enable)), int(reset)),
              "dct_plan_profile")

    def profile_read(self):
        """{kind: (ms, launches, flops, bytes)} accumulated while enabled."""
        out = {}
        for k, name in enumerate(self.KINDS):
            ms, n = C.c_double(0), C.c_int64(0)
            fl, by = C.c_double(0), C.c_double(0)
            check(lib().dct_plan_profile_get(self._h, k, C.byref(ms), C.byref(n),
                                             C.byref(fl), C.byref(by)),
                  "dct_plan_profile_get")
            out[name] = (ms.value, n.value, fl.value, by.value)
        return out

    def profile_log(self):
        """[(kind name, ms)] of every profiled launch, in launch order."""
        n = C.c_int64(0)
        check(lib().dct_plan_profile_log(self._h, 0, None, None, C.byref(n)),
              "dct_plan_profile_log")
        kinds = np.zeros(max(n.value, 1), np.int32)
        ms = np.zeros(max(n.value, 1), np.float64)
        check(lib().dct_plan_profile_log(
            self._h, n.value, kinds.ctypes.data_as(C.POINTER(C.c_int32)),
            ms.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)),
            "dct_plan_profile_log")
        return [(self.KINDS[k], float(t)) for k, t in zip(kinds[:n.value], ms[:n.value])]

    def status(self, stream):
        code, where, res = C.c_int32(0), C.c_int32(0), C.c_double(0.0)
        check(lib().dct_check_status(self._h, stream, C.byref(code),
                                     C.byref(where), C.byref(res)),
              "dct_check_status")
        return code.value, where.value, res.value

    def free(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.dct_plan_destroy(h)
        self._h = None

    def __del__(self):
        self.free()


def default_tuning(dtype):
    t = Tuning()
    check(lib().dct_tuning_default(int(dtype), C.byref(t)), "dct_tuning_default")
    return t.as_dict()
