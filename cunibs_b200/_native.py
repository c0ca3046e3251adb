"""ctypes binding of the C ABI in include/cunibs_b200.h (libcunibs_b200.so).

The library is built in-tree (cunibs_b200/_lib). There is no fallback: if it is missing or cannot
be loaded, every entry point raises.
"""

from __future__ import annotations

import ctypes as C
import weakref
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libcunibs_b200.so"
_lib: C.CDLL | None = None

OK, EINVAL, ENOMEM, ECUDA, ENOCONV, ETIMEOUT, EINTERNAL = range(7)
PREC_DEFAULT, PREC_PLAIN_FP64, PREC_MIXED, PREC_SPLIT = 0, 1, 2, 3
RECOVERY_CODES = {"raw": 0, "spr_global": 1, "spr_tissue": 2, "harmonic": 3}
SUMMARY_LEN = 16

_vp = C.c_void_p


class Params(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("min_coarse_rows", C.c_int),
        ("max_levels", C.c_int),
        ("agg_rounds", C.c_int),
        ("cheby_degree", C.c_int),
        ("cheby_lower_ratio", C.c_double),
        ("tolerance", C.c_double),
        ("max_iters", C.c_int),
        ("precision", C.c_int),
        ("inner_reduction", C.c_double),
        ("inner_max_iters", C.c_int),
        ("iters_per_sync", C.c_int),
        ("dense_max_rows", C.c_int),
    ]


class Info(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int),
        ("n_tets", C.c_int),
        ("n_skin", C.c_int),
        ("n_gray_matter", C.c_int),
        ("stiffness_nnz", C.c_longlong),
        ("ground_node", C.c_int),
        ("n_levels", C.c_int),
        ("coarse_rows", C.c_int),
        ("vcycle_levels", C.c_int),
        ("bottom_rows", C.c_int),
        ("hierarchy_builds", C.c_int),
    ]


class SolveOpts(C.Structure):
    _fields_ = [
        ("block_width", C.c_int),
        ("precision", C.c_int),
        ("tolerance", C.c_double),
        ("max_iters", C.c_int),
        ("recovery", C.c_int),
        ("warm_start", C.c_int),
    ]


class RecoveryInfo(C.Structure):
    _fields_ = [
        ("mode", C.c_int),
        ("n_slots", C.c_int),
        ("nnz", C.c_longlong),
        ("n_fallback", C.c_int),
        ("n_undetermined", C.c_int),
    ]


class BlockOut(C.Structure):
    _fields_ = [
        ("transforms", _vp),
        ("summary", _vp),
        ("iterations", _vp),
        ("relres", _vp),
        ("magnE", _vp),
        ("E", _vp),
        ("v", _vp),
        ("total_iterations", C.c_int),
        ("outer_steps", C.c_int),
        ("E_slots", _vp),
        ("warm_used", _vp),
        ("init_relres", _vp),
    ]


class NativeError(RuntimeError):
    """A failure reported by the native library (status code in ``.code``)."""

    def __init__(self, code: int, message: str) -> None:
        super().__init__(message)
        self.code = code


class ConvergenceFailure(NativeError):
    pass


def library_path() -> Path:
    return _LIB_PATH


def load() -> C.CDLL:
    """Load the native library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C cunibs_b200/csrc`"
        )
    lib = C.CDLL(str(_LIB_PATH))
    ip = C.POINTER(C.c_int)
    dp = C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    sig = {
        "cunibs_version": ([], C.c_int),
        "cunibs_last_error": ([], C.c_char_p),
        "cunibs_params_default": ([C.POINTER(Params)], C.c_int),
        "cunibs_context_create": ([dp, C.c_int, ip, ip, C.c_int, ip, C.c_int, C.POINTER(Params), C.POINTER(_vp)], C.c_int),
        "cunibs_context_destroy": ([_vp], C.c_int),
        "cunibs_context_info": ([_vp, C.POINTER(Info)], C.c_int),
        "cunibs_context_mesh": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "cunibs_context_levels": ([_vp, ip, C.c_int], C.c_int),
        "cunibs_solve_block": ([_vp, _vp, _vp, C.c_int, _vp, _vp, _vp, C.c_int, C.c_double, C.POINTER(SolveOpts), C.POINTER(BlockOut)], C.c_int),
        "cunibs_solve_block_device": ([_vp, _vp, _vp, C.c_int, _vp, _vp, _vp, C.c_int, C.c_double, C.POINTER(SolveOpts), C.POINTER(BlockOut)], C.c_int),
        "cunibs_submit_block": ([_vp, _vp, _vp, C.c_int, _vp, _vp, _vp, C.c_int, C.c_double, C.POINTER(SolveOpts),
                                 C.POINTER(C.c_longlong)], C.c_int),
        "cunibs_finish_block": ([_vp, C.c_longlong, C.POINTER(BlockOut)], C.c_int),
        "cunibs_submit_block_device": ([_vp, _vp, _vp, C.c_int, _vp, _vp, _vp, C.c_int, C.c_double,
                                        C.POINTER(SolveOpts), C.POINTER(C.c_longlong)], C.c_int),
        "cunibs_finish_block_device": ([_vp, C.c_longlong, C.POINTER(BlockOut)], C.c_int),
        "cunibs_cancel_block": ([_vp, C.c_longlong], C.c_int),
        "cunibs_context_pending": ([_vp, C.POINTER(C.c_int)], C.c_int),
        "cunibs_context_set_overlap": ([_vp, C.c_int], C.c_int),
        "cunibs_context_set_coil_table": ([_vp, C.c_int, C.c_double, C.c_double], C.c_int),
        "cunibs_context_coil_table_info": ([_vp, _vp], C.c_int),
        "cunibs_context_phase_times": ([_vp, _vp], C.c_int),
        "cunibs_context_set_conductivity": ([_vp, dp], C.c_int),
        "cunibs_context_set_conductivity_keep_coarse": ([_vp, dp], C.c_int),
        "cunibs_sigma_begin": ([_vp, _vp, _vp, C.c_int, _vp, _vp, _vp, C.c_int, C.c_double, C.POINTER(SolveOpts), dp, ip,
                                C.c_int, C.c_double, ip], C.c_int),
        "cunibs_sigma_draw": ([_vp, dp, C.POINTER(BlockOut), ip], C.c_int),
        "cunibs_sigma_end": ([_vp], C.c_int),
        "cunibs_sigma_set_guess": ([_vp, C.c_int], C.c_int),
        "cunibs_sigma_coefficients": ([C.c_int, dp, dp, ip, C.c_double, dp, ip], C.c_int),
        "cunibs_adm_create": ([_vp, ip, dp, C.c_int, dp, C.c_int, C.c_double, C.c_int, ip, dp, C.POINTER(_vp)],
                              C.c_int),
        "cunibs_adm_destroy": ([_vp], C.c_int),
        "cunibs_adm_node_weights": ([_vp, dp], C.c_int),
        "cunibs_adm_sample": ([_vp, dp, dp, ip], C.c_int),
        "cunibs_adm_qfield": ([_vp, fp, C.c_longlong], C.c_int),
        "cunibs_adm_evaluate": ([_vp, dp, dp, C.c_int, dp, C.c_int, C.c_double, dp], C.c_int),
        "cunibs_adm_evaluate_exact": ([_vp, dp, dp, C.c_int, dp, C.c_int, C.c_double, dp, dp], C.c_int),
        "cunibs_context_array": ([_vp, C.c_char_p, C.c_int, _vp, C.c_longlong, C.POINTER(C.c_longlong)], C.c_int),
        "cunibs_context_place": ([_vp, _vp, _vp, _vp, C.c_int, _vp, _vp], C.c_int),
        "cunibs_context_dadt": ([_vp, _vp, _vp, C.c_int, _vp, C.c_int, C.c_double, _vp], C.c_int),
        "cunibs_context_solve": ([_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, _vp, _vp, _vp], C.c_int),
        "cunibs_context_vcycle": ([_vp, _vp, _vp, C.c_int, C.c_int], C.c_int),
        "cunibs_select_size4": ([C.c_int, ip, ip, fp, ip, ip], C.c_int),
        "cunibs_context_summary": ([_vp, _vp, C.c_int, _vp], C.c_int),
        "cunibs_context_recovery": ([_vp, C.c_int, C.POINTER(RecoveryInfo)], C.c_int),
        "cunibs_context_recovery_array": ([_vp, C.c_int, C.c_char_p, _vp, C.c_longlong, C.POINTER(C.c_longlong)], C.c_int),
        "cunibs_context_recover": ([_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "cunibs_context_set_warmstart": ([_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "cunibs_gemm_bf16": ([_vp, C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int, C.c_int, _vp,
                              _vp, C.c_int, _vp, C.c_int, _vp], C.c_int),
        "cunibs_gemm_status": ([_vp, C.POINTER(C.c_int)], C.c_int),
        "cunibs_debug_gemm_waits": ([C.c_longlong, C.c_longlong, C.c_int], C.c_int),
        "cunibs_mlp_colsum": ([_vp, C.c_int, C.c_int, C.c_int, _vp, _vp], C.c_int),
        "cunibs_mlp_mse": ([_vp, _vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp], C.c_int),
        "cunibs_mlp_adam": ([_vp, _vp, _vp, _vp, C.c_longlong, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                             C.c_float, C.c_int, C.c_int, _vp, _vp, _vp], C.c_int),
        "cunibs_mlp_features": ([_vp, C.c_int, _vp, _vp, _vp, C.c_int, _vp], C.c_int),
        "cunibs_context_set_timing": ([_vp, C.c_int], C.c_int),
        "cunibs_context_stage_times": ([_vp, dp, C.c_int], C.c_int),
        "cunibs_context_stream": ([_vp, C.POINTER(_vp)], C.c_int),
        "cunibs_kernel_launches": ([], C.c_longlong),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc == OK:
        return
    msg = load().cunibs_last_error().decode(errors="replace")
    if rc == EINVAL:
        raise ValueError(msg)
    if rc == ENOCONV:
        raise ConvergenceFailure(rc, msg)
    if rc == ENOMEM:
        raise MemoryError(msg)
    raise NativeError(rc, msg)


def _guess_code(warm_start) -> int:
    """cunibs_solve_opts.warm_start: False/0 none, True/1 the network, "projection"/2 the Galerkin
    projection onto the network's basis."""
    if warm_start == "projection":
        return 2
    code = int(warm_start)
    if code not in (0, 1, 2):
        raise ValueError("warm_start must be False, True or 'projection'")
    return code


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_vp)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def default_params() -> Params:
    p = Params()
    check(load().cunibs_params_default(C.byref(p)))
    return p


# Names of the int32 arrays cunibs_context_array serves; the rest are float64.
_INT_ARRAYS = {
    "node_perm", "tet_perm", "tet_nodes", "tet_tags", "skin_tris", "n2c_ptr", "n2c_idx", "stiff_ptr",
    "stiff_col", "gm_index", "a_ptr", "a_col", "agg", "p_ptr", "p_col", "coarse_ptr", "coarse_col",
}


class Context:
    """One subject's device state: a handle from cunibs_context_create."""

    def __init__(self, nodes_mm, tet_nodes, tet_tags, skin_tris, params: Params | None = None) -> None:
        lib = load()
        nodes = np.ascontiguousarray(nodes_mm, dtype=np.float64).reshape(-1, 3)
        tets = np.ascontiguousarray(tet_nodes, dtype=np.int32).reshape(-1, 4)
        tags = np.ascontiguousarray(tet_tags, dtype=np.int32).reshape(-1)
        skin = np.ascontiguousarray(skin_tris, dtype=np.int32).reshape(-1, 3)
        if skin.size == 0:
            skin = np.zeros((1, 3), np.int32)[:0]
        h = _vp()
        prm = params if params is not None else default_params()
        check(lib.cunibs_context_create(
            nodes.ctypes.data_as(C.POINTER(C.c_double)), nodes.shape[0], _ip(tets), _ip(tags), tets.shape[0],
            _ip(skin) if skin.shape[0] else None, skin.shape[0], C.byref(prm), C.byref(h)))
        self._h = h
        self._lib = lib
        self._submitted: dict[int, tuple] = {}
        self._study: tuple | None = None
        self._adms: weakref.WeakSet = weakref.WeakSet()
        self.params = prm
        info = Info()
        check(lib.cunibs_context_info(h, C.byref(info)))
        self.n_nodes = info.n_nodes
        self.n_tets = info.n_tets
        self.n_skin = info.n_skin
        self.n_gray_matter = info.n_gray_matter
        self.stiffness_nnz = info.stiffness_nnz
        self.ground_node = info.ground_node
        self.n_levels = info.n_levels
        self.coarse_rows = info.coarse_rows
        self.vcycle_levels = info.vcycle_levels
        self.bottom_rows = info.bottom_rows

    @property
    def hierarchy_builds(self) -> int:
        """AMG hierarchy builds over the context's life (1 at create; each rebuild adds one)."""
        info = Info()
        check(self._lib.cunibs_context_info(self.handle, C.byref(info)))
        return int(info.hierarchy_builds)

    def close(self) -> None:
        # Handles that live on this context (auxiliary-dipole-method state) go first.
        for a in list(getattr(self, "_adms", ())):
            a.close()
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.cunibs_context_destroy(h)
            self._h = _vp()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter teardown
            pass

    @property
    def handle(self):
        if not self._h.value:
            raise ValueError("the context has been freed")
        return self._h

    def mesh(self):
        nodes = np.empty((self.n_nodes, 3))
        tets = np.empty((self.n_tets, 4), np.int32)
        tags = np.empty(self.n_tets, np.int32)
        skin = np.empty((max(self.n_skin, 1), 3), np.int32)
        node_perm = np.empty(self.n_nodes, np.int32)
        tet_perm = np.empty(self.n_tets, np.int32)
        check(self._lib.cunibs_context_mesh(self.handle, _p(nodes), _p(tets), _p(tags), _p(skin), _p(node_perm), _p(tet_perm)))
        return nodes, tets, tags, skin[: self.n_skin], node_perm, tet_perm

    def levels(self) -> list[int]:
        out = np.empty(64, np.int32)
        check(self._lib.cunibs_context_levels(self.handle, _ip(out), 64))
        return out[: self.n_levels + 1].tolist()

    def array(self, name: str, level: int = -1) -> np.ndarray:
        n = C.c_longlong()
        check(self._lib.cunibs_context_array(self.handle, name.encode(), level, None, 0, C.byref(n)))
        dt = np.int32 if name in _INT_ARRAYS else np.float64
        out = np.empty(n.value, dt)
        check(self._lib.cunibs_context_array(self.handle, name.encode(), level, _p(out), n.value, C.byref(n)))
        return out

    def place(self, centers, handles, dists):
        centers = np.ascontiguousarray(centers, np.float64).reshape(-1, 3)
        k = centers.shape[0]
        handles_a = None if handles is None else np.ascontiguousarray(handles, np.float64).reshape(-1, 3)
        dists = np.ascontiguousarray(dists, np.float64).reshape(-1)
        T = np.empty((k, 4, 4))
        deg = np.empty(k, np.int32)
        check(self._lib.cunibs_context_place(self.handle, _p(centers), _p(handles_a), _p(dists), k, _p(T), _p(deg)))
        return T, deg

    def dadt(self, coil, transforms, didt) -> np.ndarray:
        T = np.ascontiguousarray(transforms, np.float64).reshape(-1, 16)
        k = T.shape[0]
        pos = np.ascontiguousarray(coil.positions_m, np.float64)
        mom = np.ascontiguousarray(coil.moments, np.float64)
        out = np.empty((k, self.n_nodes, 3), np.float32)
        check(self._lib.cunibs_context_dadt(self.handle, _p(pos), _p(mom), pos.shape[0], _p(T), k, float(didt), _p(out)))
        return out

    def solve(self, B, k, width, precision=PREC_DEFAULT, tolerance=0.0, max_iters=0, x0=None):
        B = np.ascontiguousarray(B, np.float64)
        X = np.empty_like(B)
        it = np.empty(k, np.int32)
        rel = np.empty(k)
        x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        check(self._lib.cunibs_context_solve(self.handle, _p(B), _p(X), k, width, precision, float(tolerance),
                                             int(max_iters), _p(x0a), _p(it), _p(rel)))
        return X, it, rel

    def vcycle(self, r, fp32=False) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        k = 1 if r.ndim == 1 else r.shape[1]
        z = np.empty_like(r)
        check(self._lib.cunibs_context_vcycle(self.handle, _p(r), _p(z), k, int(bool(fp32))))
        return z

    def summary(self, magnE) -> np.ndarray:
        m = np.ascontiguousarray(magnE, np.float32).reshape(-1, self.n_tets)
        out = np.empty((m.shape[0], SUMMARY_LEN))
        check(self._lib.cunibs_context_summary(self.handle, _p(m), m.shape[0], _p(out)))
        return out

    def recovery(self, mode: str) -> dict:
        """Build (once) the recovery operator of ``mode`` and return its counts."""
        info = RecoveryInfo()
        check(self._lib.cunibs_context_recovery(self.handle, RECOVERY_CODES[mode], C.byref(info)))
        return {"mode": mode, "n_slots": info.n_slots, "nnz": info.nnz, "n_fallback": info.n_fallback,
                "n_undetermined": info.n_undetermined}

    def recovery_array(self, mode: str, name: str) -> np.ndarray:
        code = RECOVERY_CODES[mode]
        n = C.c_longlong()
        check(self._lib.cunibs_context_recovery_array(self.handle, code, name.encode(), None, 0, C.byref(n)))
        out = np.empty(n.value, np.float32 if name == "w" else np.int32)
        check(self._lib.cunibs_context_recovery_array(self.handle, code, name.encode(), _p(out), n.value, C.byref(n)))
        return out.reshape(-1, 3) if (name == "w" and mode == "harmonic") else out

    def recover(self, mode: str, *, v=None, dadt_nodes=None, elements=None):
        """cunibs_context_recover on host data: (E_slots (k,S,3), E (k,M,3), magnE (k,M))."""
        info = self.recovery(mode)
        va = da = ea = None
        if mode == "harmonic":
            va = np.ascontiguousarray(v, np.float64).reshape(-1, self.n_nodes)
            da = np.ascontiguousarray(dadt_nodes, np.float32).reshape(-1, self.n_nodes, 3)
            k = va.shape[0]
        else:
            ea = np.ascontiguousarray(elements, np.float32).reshape(-1, self.n_tets, 3)
            k = ea.shape[0]
        slots = np.empty((k, info["n_slots"], 3), np.float32)
        E = np.empty((k, self.n_tets, 3), np.float32)
        mag = np.empty((k, self.n_tets), np.float32)
        check(self._lib.cunibs_context_recover(self.handle, RECOVERY_CODES[mode], k, _p(va), _p(da), _p(ea),
                                               _p(slots), _p(E), _p(mag)))
        return slots, E, mag

    def set_warm_start(self, depth, hidden, n_out, weights, biases, feature_mean, feature_std, coef_mean, coef_std,
                       basis) -> None:
        """Install a trained warm-start network (device pointers as ints); weights=None removes it."""
        if weights is None:
            check(self._lib.cunibs_context_set_warmstart(self.handle, 0, 0, 0, None, None, None, None, None, None, None))
            return
        w = (_vp * len(weights))(*weights)
        b = (_vp * len(biases))(*biases)
        check(self._lib.cunibs_context_set_warmstart(self.handle, int(depth), int(hidden), int(n_out), w, b,
                                                     feature_mean, feature_std, coef_mean, coef_std, basis))

    def set_timing(self, on: bool = True) -> None:
        check(self._lib.cunibs_context_set_timing(self.handle, int(bool(on))))

    def stage_times(self) -> np.ndarray:
        ms = np.empty(5)
        check(self._lib.cunibs_context_stage_times(self.handle, ms.ctypes.data_as(C.POINTER(C.c_double)), 5))
        return ms

    def stream(self) -> int:
        out = _vp()
        check(self._lib.cunibs_context_stream(self.handle, C.byref(out)))
        return int(out.value or 0)

    def solve_block_device(self, pos, mom, n_dip, centers, handles, dists, k, didt, out_ptrs, *, block_width=0,
                           precision=PREC_DEFAULT, tolerance=0.0, max_iters=0, recovery="raw",
                           warm_start=False) -> tuple[int, int]:
        """cunibs_solve_block_device on raw device pointers (ints); out_ptrs maps output names to pointers."""
        out = BlockOut(out_ptrs.get("transforms"), out_ptrs.get("summary"), out_ptrs.get("iterations"),
                       out_ptrs.get("relres"), out_ptrs.get("magnE"), out_ptrs.get("E"), out_ptrs.get("v"), 0, 0,
                       out_ptrs.get("E_slots"), out_ptrs.get("warm_used"), out_ptrs.get("init_relres"))
        opts = SolveOpts(int(block_width), int(precision), float(tolerance), int(max_iters), RECOVERY_CODES[recovery],
                         _guess_code(warm_start))
        check(self._lib.cunibs_solve_block_device(self.handle, pos, mom, int(n_dip), centers, handles, dists, int(k),
                                                  float(didt), C.byref(opts), C.byref(out)))
        return out.total_iterations, out.outer_steps

    def submit_block_device(self, pos, mom, n_dip, centers, handles, dists, k, didt, *, block_width=0,
                            precision=PREC_DEFAULT, tolerance=0.0, max_iters=0, recovery="raw",
                            warm_start=False) -> int:
        """cunibs_submit_block_device: prepare a block on raw device pointers (ints) without waiting;
        returns its ticket."""
        opts = SolveOpts(int(block_width), int(precision), float(tolerance), int(max_iters), RECOVERY_CODES[recovery],
                         _guess_code(warm_start))
        t = C.c_longlong(0)
        check(self._lib.cunibs_submit_block_device(self.handle, pos, mom, int(n_dip), centers, handles, dists, int(k),
                                                   float(didt), C.byref(opts), C.byref(t)))
        return t.value

    def finish_block_device(self, ticket: int, out_ptrs) -> tuple[int, int]:
        """cunibs_finish_block_device: solve a submitted block into out_ptrs (device pointers)."""
        out = BlockOut(out_ptrs.get("transforms"), out_ptrs.get("summary"), out_ptrs.get("iterations"),
                       out_ptrs.get("relres"), out_ptrs.get("magnE"), out_ptrs.get("E"), out_ptrs.get("v"), 0, 0,
                       out_ptrs.get("E_slots"), out_ptrs.get("warm_used"), out_ptrs.get("init_relres"))
        check(self._lib.cunibs_finish_block_device(self.handle, int(ticket), C.byref(out)))
        return out.total_iterations, out.outer_steps

    @property
    def pending(self) -> int:
        n = C.c_int(0)
        check(self._lib.cunibs_context_pending(self.handle, C.byref(n)))
        return n.value

    def set_overlap(self, blocks_per_sm: int) -> None:
        check(self._lib.cunibs_context_set_overlap(self.handle, int(blocks_per_sm)))

    def set_coil_table(self, enabled: bool = True, near_mm: float = 15.0, step: float = 0.035) -> None:
        """cunibs_context_set_coil_table: the block entries read the coil's field from a table sampled
        once per coil for nodes deeper than near_mm below the coil (enabled), or sum every dipole at
        every node (not enabled)."""
        check(self._lib.cunibs_context_set_coil_table(self.handle, 1 if enabled else 0, float(near_mm), float(step)))

    def phase_times(self) -> list[float]:
        """cunibs_context_phase_times: host milliseconds to the end of each phase of the last
        cunibs_sigma_begin."""
        out = np.zeros(8, np.float64)
        check(self._lib.cunibs_context_phase_times(self.handle, out.ctypes.data))
        return [round(float(v), 3) for v in out]

    def coil_table_info(self) -> dict:
        """cunibs_context_coil_table_info as a dict."""
        out = np.zeros(8, np.float64)
        check(self._lib.cunibs_context_coil_table_info(self.handle, out.ctypes.data))
        return {"mode": int(out[0]), "in_use": bool(out[1]), "points": int(out[2]), "layers": int(out[3]),
                "check_rel_l2": float(out[4]), "builds": int(out[5]), "last_near_nodes": int(out[6]),
                "last_node_placements": int(out[7])}

    def set_conductivity(self, sigma_by_tag, *, keep_coarse: bool = False) -> None:
        """New conductivities (index = tissue tag). keep_coarse: refresh only the finest AMG level
        (cunibs_context_set_conductivity_keep_coarse), the cheap per-sample step of a Monte Carlo."""
        s = np.ascontiguousarray(sigma_by_tag, np.float64).reshape(11)
        fn = (self._lib.cunibs_context_set_conductivity_keep_coarse if keep_coarse
              else self._lib.cunibs_context_set_conductivity)
        check(fn(self.handle, s.ctypes.data_as(C.POINTER(C.c_double))))

    def sigma_begin(self, coil, centers, handles, dists, didt, sigma_nominal, tags, *, sensitivity_tol=1e-3,
                    precision=PREC_DEFAULT, tolerance=0.0, max_iters=0, magnitude=False, vectors=False,
                    potential=False, recovery="raw", nodal=False) -> np.ndarray:
        """cunibs_sigma_begin: open a conductivity study of one block of placements; the outputs of
        every draw are chosen here. Returns the sensitivity-subspace rank per placement."""
        pos, mom, centers, handles, dists = self._block_inputs(coil, centers, handles, dists)
        k = centers.shape[0]
        if nodal and recovery == "raw":
            raise ValueError("nodal=True needs a recovery mode")
        opts = SolveOpts(0, int(precision), float(tolerance), int(max_iters), RECOVERY_CODES[recovery], 0)
        sig = np.ascontiguousarray(sigma_nominal, np.float64).reshape(11)
        tg = np.ascontiguousarray(tags, np.int32).reshape(-1)
        rank = np.zeros(k, np.int32)
        check(self._lib.cunibs_sigma_begin(self.handle, _p(pos), _p(mom), pos.shape[0], _p(centers), _p(handles),
                                           _p(dists), k, float(didt), C.byref(opts),
                                           sig.ctypes.data_as(C.POINTER(C.c_double)), _ip(tg), tg.shape[0],
                                           float(sensitivity_tol), _ip(rank)))
        self._study = (k, tg.shape[0], magnitude, vectors, potential, recovery, nodal)
        return rank

    def sigma_draw(self, sigma) -> dict:
        """cunibs_sigma_draw: one draw (the perturbed tissues' conductivities, in the study's tag
        order); the same dict as solve_block plus "resetup" (1 when the draw needed its own hierarchy)."""
        if self._study is None:
            raise ValueError("no conductivity study is open")
        k, n_tags, magnitude, vectors, potential, recovery, nodal = self._study
        s = np.ascontiguousarray(sigma, np.float64).reshape(n_tags)
        res, out = self._block_outputs(k, magnitude, vectors, potential, recovery, nodal)
        flag = C.c_int(0)
        check(self._lib.cunibs_sigma_draw(self.handle, s.ctypes.data_as(C.POINTER(C.c_double)), C.byref(out),
                                          C.byref(flag)))
        res["total_iterations"] = out.total_iterations
        res["outer_steps"] = out.outer_steps
        res["resetup"] = flag.value
        return res

    def sigma_set_guess(self, mode: str) -> None:
        """cunibs_sigma_set_guess: the initial guess of the following draws ("subspace", the default;
        "nominal", the nominal potential alone; "zero")."""
        codes = {"subspace": 0, "nominal": 1, "zero": 2}
        if mode not in codes:
            raise ValueError("guess mode must be 'subspace', 'nominal' or 'zero'")
        check(self._lib.cunibs_sigma_set_guess(self.handle, codes[mode]))

    def sigma_end(self) -> None:
        """cunibs_sigma_end: close the study; the context is back at the nominal conductivities."""
        self._study = None
        check(self._lib.cunibs_sigma_end(self.handle))

    @staticmethod
    def _block_inputs(coil, centers, handles, dists):
        centers = np.ascontiguousarray(centers, np.float64).reshape(-1, 3)
        handles = np.ascontiguousarray(handles, np.float64).reshape(-1, 3)
        dists = np.ascontiguousarray(dists, np.float64).reshape(-1)
        pos = np.ascontiguousarray(coil.positions_m, np.float64)
        mom = np.ascontiguousarray(coil.moments, np.float64)
        return pos, mom, centers, handles, dists

    def _block_outputs(self, k, magnitude, vectors, potential, recovery, nodal):
        res = {
            "transform": np.empty((k, 4, 4)),
            "summary": np.empty((k, SUMMARY_LEN)),
            "iterations": np.empty(k, np.int32),
            "relative_residual": np.empty(k),
            "magnE": np.empty((k, self.n_tets), np.float32) if magnitude else None,
            "E": np.empty((k, self.n_tets, 3), np.float32) if vectors else None,
            "v": np.empty((k, self.n_nodes)) if potential else None,
            "E_slots": None,
            "warm_used": np.zeros(k, np.int32),
            "init_relres": np.ones(k),
        }
        if nodal:
            if recovery == "raw":
                raise ValueError("nodal=True needs a recovery mode")
            res["E_slots"] = np.empty((k, self.recovery(recovery)["n_slots"], 3), np.float32)
        out = BlockOut(_p(res["transform"]), _p(res["summary"]), _p(res["iterations"]), _p(res["relative_residual"]),
                       _p(res["magnE"]), _p(res["E"]), _p(res["v"]), 0, 0, _p(res["E_slots"]), _p(res["warm_used"]),
                       _p(res["init_relres"]))
        return res, out

    def solve_block(self, coil, centers, handles, dists, didt, *, block_width=0, precision=PREC_DEFAULT,
                    tolerance=0.0, max_iters=0, magnitude=False, vectors=False, potential=False,
                    recovery="raw", nodal=False, warm_start=False) -> dict:
        """One block of k placements through cunibs_solve_block (host buffers in and out)."""
        pos, mom, centers, handles, dists = self._block_inputs(coil, centers, handles, dists)
        k = centers.shape[0]
        res, out = self._block_outputs(k, magnitude, vectors, potential, recovery, nodal)
        opts = SolveOpts(int(block_width), int(precision), float(tolerance), int(max_iters), RECOVERY_CODES[recovery],
                         _guess_code(warm_start))
        check(self._lib.cunibs_solve_block(self.handle, _p(pos), _p(mom), pos.shape[0], _p(centers), _p(handles),
                                           _p(dists), k, float(didt), C.byref(opts), C.byref(out)))
        res["total_iterations"] = out.total_iterations
        res["outer_steps"] = out.outer_steps
        return res

    def submit_block(self, coil, centers, handles, dists, didt, *, block_width=0, precision=PREC_DEFAULT,
                     tolerance=0.0, max_iters=0, magnitude=False, vectors=False, potential=False,
                     recovery="raw", nodal=False, warm_start=False) -> int:
        """cunibs_submit_block: prepare a block (host inputs, copied now) without waiting for the
        work; returns the ticket that finish_block takes. The outputs are chosen here."""
        pos, mom, centers, handles, dists = self._block_inputs(coil, centers, handles, dists)
        k = centers.shape[0]
        if nodal and recovery == "raw":
            raise ValueError("nodal=True needs a recovery mode")
        opts = SolveOpts(int(block_width), int(precision), float(tolerance), int(max_iters), RECOVERY_CODES[recovery],
                         _guess_code(warm_start))
        t = C.c_longlong(0)
        check(self._lib.cunibs_submit_block(self.handle, _p(pos), _p(mom), pos.shape[0], _p(centers), _p(handles),
                                            _p(dists), k, float(didt), C.byref(opts), C.byref(t)))
        self._submitted[t.value] = (k, magnitude, vectors, potential, recovery, nodal)
        return t.value

    def cancel_block(self, ticket: int) -> None:
        """cunibs_cancel_block: drop a submitted block without solving it."""
        self._submitted.pop(ticket, None)
        check(self._lib.cunibs_cancel_block(self.handle, int(ticket)))

    def finish_block(self, ticket: int) -> dict:
        """cunibs_finish_block: solve a submitted block; the same dict as solve_block."""
        k, magnitude, vectors, potential, recovery, nodal = self._submitted.pop(ticket)
        res, out = self._block_outputs(k, magnitude, vectors, potential, recovery, nodal)
        check(self._lib.cunibs_finish_block(self.handle, int(ticket), C.byref(out)))
        res["total_iterations"] = out.total_iterations
        res["outer_steps"] = out.outer_steps
        return res


def kernel_launches() -> int:
    return int(load().cunibs_kernel_launches())


class Adm:
    """An auxiliary-dipole-method handle (cunibs_adm_*): the adjoint state of one target functional
    on a context, and the reciprocity field it last sampled. The context must stay open."""

    def __init__(self, ctx: Context, elem_idx, weights, directions, tolerance: float, max_iters: int) -> None:
        lib = load()
        idx = np.ascontiguousarray(elem_idx, np.int32).reshape(-1)
        w = np.ascontiguousarray(weights, np.float64).reshape(-1)
        d = np.ascontiguousarray(directions, np.float64).reshape(-1, 3)
        if idx.shape != w.shape:
            raise ValueError("elem_idx and weights must have the same length")
        self.n_dir = d.shape[0]
        self.n_nodes = ctx.n_nodes
        self.iterations = np.zeros(self.n_dir, np.int32)
        self.relres = np.zeros(self.n_dir)
        h = _vp()
        dp = C.POINTER(C.c_double)
        check(lib.cunibs_adm_create(ctx.handle, _ip(idx), w.ctypes.data_as(dp), idx.shape[0], d.ctypes.data_as(dp),
                                    self.n_dir, float(tolerance), int(max_iters), _ip(self.iterations),
                                    self.relres.ctypes.data_as(dp), C.byref(h)))
        self._h = h
        self._lib = lib
        self._ctx = ctx  # keeps the context object alive; closing the context closes this handle first
        ctx._adms.add(self)
        self.shape: tuple[int, int, int] | None = None
        self.sample_id = 0

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            check(self._lib.cunibs_adm_destroy(self._h))
            self._h = _vp()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if not self._h.value:
            raise ValueError("the auxiliary-dipole-method handle has been closed (or its context freed)")
        return self._h

    def node_weights(self) -> np.ndarray:
        out = np.empty((self.n_dir, self.n_nodes, 3))
        check(self._lib.cunibs_adm_node_weights(self.handle, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def sample(self, origin_mm, spacing_mm, shape) -> int:
        o = np.ascontiguousarray(origin_mm, np.float64).reshape(3)
        sp = np.ascontiguousarray(spacing_mm, np.float64).reshape(3)
        sh = np.ascontiguousarray(shape, np.int32).reshape(3)
        dp = C.POINTER(C.c_double)
        check(self._lib.cunibs_adm_sample(self.handle, o.ctypes.data_as(dp), sp.ctypes.data_as(dp), _ip(sh)))
        self.shape = tuple(int(v) for v in sh)
        self.sample_id += 1
        return self.sample_id

    def qfield(self) -> np.ndarray:
        if self.shape is None:
            raise ValueError("the reciprocity field has not been sampled")
        out = np.empty((self.n_dir, *self.shape, 3), np.float32)
        check(self._lib.cunibs_adm_qfield(self.handle, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def _eval(self, fn, coil, transforms, didt, *extra) -> np.ndarray:
        T = np.ascontiguousarray(transforms, np.float64).reshape(-1, 16)
        pos = np.ascontiguousarray(coil.positions_m, np.float64)
        mom = np.ascontiguousarray(coil.moments, np.float64)
        out = np.empty((T.shape[0], self.n_dir))
        dp = C.POINTER(C.c_double)
        check(fn(self.handle, pos.ctypes.data_as(dp), mom.ctypes.data_as(dp), pos.shape[0], T.ctypes.data_as(dp),
                 T.shape[0], float(didt), *extra, out.ctypes.data_as(dp)))
        return out

    def evaluate(self, coil, transforms, didt) -> np.ndarray:
        return self._eval(self._lib.cunibs_adm_evaluate, coil, transforms, didt)

    def evaluate_exact(self, coil, transforms, didt, center_mm=None) -> np.ndarray:
        c = None if center_mm is None else np.ascontiguousarray(center_mm, np.float64).reshape(3)
        cp_ = None if c is None else c.ctypes.data_as(C.POINTER(C.c_double))
        return self._eval(self._lib.cunibs_adm_evaluate_exact, coil, transforms, didt, cp_)


def sigma_coefficients(gram, proj, active, rtol: float = 1e-12):
    """cunibs_sigma_coefficients (host only): the draw-coefficient map Z of one placement and the
    rank of its sensitivity subspace."""
    lib = load()
    g = np.ascontiguousarray(gram, np.float64)
    n = g.shape[0]
    pr = np.ascontiguousarray(proj, np.float64).reshape(n, n)
    act = np.ascontiguousarray(active, np.int32).reshape(n)
    z = np.empty((n, n))
    rank = C.c_int()
    dp = C.POINTER(C.c_double)
    check(lib.cunibs_sigma_coefficients(n, g.ctypes.data_as(dp), pr.ctypes.data_as(dp), _ip(act), float(rtol),
                                        z.ctypes.data_as(dp), C.byref(rank)))
    return z, rank.value


def select_size4(row_ptr, col_idx, values):
    lib = load()
    rp = np.ascontiguousarray(row_ptr, np.int32)
    n = rp.shape[0] - 1
    agg = np.empty(max(n, 1), np.int32)
    nc = C.c_int()
    ci = np.ascontiguousarray(col_idx, np.int32)
    va = np.ascontiguousarray(values, np.float32)
    check(lib.cunibs_select_size4(n, _ip(rp), _ip(ci), va.ctypes.data_as(C.POINTER(C.c_float)), _ip(agg), C.byref(nc)))
    return agg[:n], nc.value
