"""ctypes binding of the CPU oracle library (oracle/_build/liboracle.so). Test infrastructure."""

from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "liboracle.so"
_lib: C.CDLL | None = None

SUMMARY_LEN = 16
RECOVERY_CODES = {"raw": 0, "spr_global": 1, "spr_tissue": 2, "harmonic": 3}
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class _Params(C.Structure):
    _fields_ = [
        ("min_coarse_rows", C.c_int),
        ("max_levels", C.c_int),
        ("agg_rounds", C.c_int),
        ("cheby_degree", C.c_int),
        ("cheby_lower_ratio", C.c_double),
        ("n_threads", C.c_int),
        ("has_sigma", C.c_int),
        ("sigma_by_tag", C.c_double * 11),
    ]


@dataclass
class OracleParams:
    min_coarse_rows: int = 128
    max_levels: int = 50
    agg_rounds: int = 2
    cheby_degree: int = 2
    cheby_lower_ratio: float = 12.0
    n_threads: int = 0
    sigma_by_tag: tuple[float, ...] | None = None  # 11 entries indexed by tag: a conductivity draw


def build_oracle() -> Path:
    """Compile the oracle library with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def _load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        build_oracle()
    lib = C.CDLL(str(_LIB_PATH))
    lib.orc_ctx_create.restype = C.c_void_p
    lib.orc_ctx_create.argtypes = [_dp, C.c_int, _ip, _ip, C.c_int, _ip, C.c_int, C.POINTER(_Params), C.c_char_p, C.c_int]
    lib.orc_ctx_destroy.argtypes = [C.c_void_p]
    lib.orc_n_levels.argtypes = [C.c_void_p]
    lib.orc_get_i32.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.c_long)]
    lib.orc_get_f64.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_long)]
    lib.orc_vcycle_apply.argtypes = [C.c_void_p, _dp, _dp, C.c_int]
    vp = C.c_void_p
    lib.orc_solve.argtypes = [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double, C.c_int,
                              C.c_int, vp, vp, vp, vp, vp, vp, vp, C.c_char_p, C.c_int]
    lib.orc_recovery_build.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_int]
    lib.orc_recovery_i32.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.c_long)]
    lib.orc_recovery_w.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_long)]
    lib.orc_recovery_apply.argtypes = [C.c_void_p, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
    lib.orc_select_size4.argtypes = [C.c_int, _ip, _ip, _fp, _ip]
    lib.orc_select_size4.restype = C.c_int
    lib.orc_l1_dinv_f32.argtypes = [C.c_int, _ip, _ip, _fp, _fp]
    lib.orc_dadt.argtypes = [_dp, _dp, C.c_int, _dp, C.c_double, _dp, C.c_int, _dp]
    lib.orc_place.argtypes = [C.c_void_p, _dp, vp, _dp, C.c_int, _dp, _ip]
    lib.orc_summary.argtypes = [_fp, _fp, _dp, _ip, C.c_int, C.c_int, _dp]
    lib.orc_weighted_quantiles.argtypes = [_dp, _dp, C.c_int, _dp, C.c_int, _dp]
    _lib = lib
    return lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """FP64 CPU restatement of one subject's solver state."""

    def __init__(self, mesh, params: OracleParams | None = None) -> None:
        lib = _load()
        p = params or OracleParams()
        sig = (C.c_double * 11)(*(p.sigma_by_tag if p.sigma_by_tag is not None else [0.0] * 11))
        cp = _Params(p.min_coarse_rows, p.max_levels, p.agg_rounds, p.cheby_degree, p.cheby_lower_ratio, p.n_threads,
                     1 if p.sigma_by_tag is not None else 0, sig)
        err = C.create_string_buffer(512)
        nodes = np.ascontiguousarray(mesh.nodes_mm, dtype=np.float64)
        tets = np.ascontiguousarray(mesh.tet_nodes, dtype=np.int32)
        tags = np.ascontiguousarray(mesh.tet_tags, dtype=np.int32)
        skin = np.ascontiguousarray(mesh.skin_tris, dtype=np.int32).reshape(-1, 3)
        if skin.size == 0:
            skin = np.zeros((0, 3), np.int32)
        h = lib.orc_ctx_create(nodes, nodes.shape[0], tets, tags, tets.shape[0], skin, skin.shape[0], C.byref(cp), err, 512)
        if not h:
            raise ValueError(err.value.decode())
        self._h = h
        self._lib = lib
        self.n_nodes = int(nodes.shape[0])
        self.n_tets = int(tets.shape[0])

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            self._lib.orc_ctx_destroy(h)
            self._h = None

    @property
    def n_levels(self) -> int:
        return int(self._lib.orc_n_levels(self._h))

    def i32(self, name: str, level: int = -1) -> np.ndarray:
        p = C.POINTER(C.c_int)()
        n = C.c_long()
        if self._lib.orc_get_i32(self._h, name.encode(), level, C.byref(p), C.byref(n)) != 0:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.empty(0, np.int32)

    def f64(self, name: str, level: int = -1) -> np.ndarray:
        p = C.POINTER(C.c_double)()
        n = C.c_long()
        if self._lib.orc_get_f64(self._h, name.encode(), level, C.byref(p), C.byref(n)) != 0:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.empty(0)

    def vcycle(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, dtype=np.float64)
        k = 1 if r.ndim == 1 else r.shape[1]
        z = np.empty_like(r)
        self._lib.orc_vcycle_apply(self._h, r, z, k)
        return z

    def place(self, centers, handles, dists):
        centers = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        k = centers.shape[0]
        handles_a = None if handles is None else np.ascontiguousarray(handles, dtype=np.float64).reshape(-1, 3)
        dists = np.ascontiguousarray(dists, dtype=np.float64).reshape(-1)
        T = np.empty((k, 16))
        deg = np.empty(k, np.int32)
        if self._lib.orc_place(self._h, centers, _ptr(handles_a), dists, k, T, deg) != 0:
            raise ValueError("placement failed")
        return T.reshape(k, 4, 4), deg

    def recovery(self, mode: str) -> dict:
        """Build (once) and return a recovery operator's arrays and counts."""
        code = RECOVERY_CODES[mode]
        err = C.create_string_buffer(512)
        if self._lib.orc_recovery_build(self._h, code, err, 512) != 0:
            raise ValueError(err.value.decode())
        out = {}
        for name in ("ptr", "idx", "slot_of_corner", "slot_node", "slot_tag", "status", "is_boundary", "counts"):
            p = C.POINTER(C.c_int)()
            n = C.c_long()
            if self._lib.orc_recovery_i32(self._h, code, name.encode(), C.byref(p), C.byref(n)) != 0:
                raise KeyError(name)
            out[name] = np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.empty(0, np.int32)
        pw = C.POINTER(C.c_float)()
        n = C.c_long()
        self._lib.orc_recovery_w(self._h, code, C.byref(pw), C.byref(n))
        w = np.ctypeslib.as_array(pw, shape=(n.value,)).copy() if n.value else np.empty(0, np.float32)
        out["w"] = w.reshape(-1, 3) if mode == "harmonic" else w
        out["n_slots"], out["n_fallback"], out["n_undetermined"] = (int(x) for x in out.pop("counts"))
        return out

    def recovery_apply(self, mode: str, *, v=None, dadt_nodes=None, elements=None):
        """The CUDA apply kernels' arithmetic on given inputs: (E_slots, E, magnE), k columns."""
        code = RECOVERY_CODES[mode]
        op = self.recovery(mode)
        if mode == "harmonic":
            v = np.ascontiguousarray(v, np.float64).reshape(-1, self.n_nodes)
            dadt_nodes = np.ascontiguousarray(dadt_nodes, np.float32).reshape(-1, self.n_nodes, 3)
            k = v.shape[0]
        else:
            elements = np.ascontiguousarray(elements, np.float32).reshape(-1, self.n_tets, 3)
            k = elements.shape[0]
        slots = np.empty((k, op["n_slots"], 3), np.float32)
        E = np.empty((k, self.n_tets, 3), np.float32)
        mag = np.empty((k, self.n_tets), np.float32)
        self._lib.orc_recovery_apply(self._h, code, k, _ptr(v), _ptr(dadt_nodes), _ptr(elements), _ptr(slots),
                                     _ptr(E), _ptr(mag))
        return slots, E, mag

    def solve(self, coil, centers, handles, dists, didt=1e6, tolerance=1e-10, max_iters=2000, recovery="raw"):
        """Full pipeline for k placements; returns a dict of per-placement arrays."""
        centers = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        handles = np.ascontiguousarray(handles, dtype=np.float64).reshape(-1, 3)
        dists = np.ascontiguousarray(dists, dtype=np.float64).reshape(-1)
        k = centers.shape[0]
        pos = np.ascontiguousarray(coil.positions_m, dtype=np.float64)
        mom = np.ascontiguousarray(coil.moments, dtype=np.float64)
        T = np.empty((k, 16))
        v = np.empty((k, self.n_nodes))
        mag = np.empty((k, self.n_tets), np.float32)
        E = np.empty((k, self.n_tets, 3), np.float32)
        S = np.empty((k, SUMMARY_LEN))
        it = np.empty(k, np.int32)
        rel = np.empty(k)
        err = C.create_string_buffer(512)
        rc = self._lib.orc_solve(self._h, pos, mom, pos.shape[0], centers, handles, dists, k, float(didt), float(tolerance),
                                 int(max_iters), RECOVERY_CODES[recovery], _ptr(T), _ptr(v), _ptr(mag), _ptr(E), _ptr(S), _ptr(it), _ptr(rel), err, 512)
        if rc != 0:
            raise ValueError(err.value.decode())
        return {"transform": T.reshape(k, 4, 4), "v": v, "magnE": mag, "E": E, "summary": S, "iterations": it, "relative_residual": rel}


def oracle_select_size4(row_ptr, col_idx, values) -> tuple[np.ndarray, int]:
    lib = _load()
    rp = np.ascontiguousarray(row_ptr, np.int32)
    n = rp.shape[0] - 1
    agg = np.empty(n, np.int32)
    nc = lib.orc_select_size4(n, rp, np.ascontiguousarray(col_idx, np.int32), np.ascontiguousarray(values, np.float32), agg)
    return agg, int(nc)


def oracle_l1_dinv_f32(row_ptr, col_idx, values) -> np.ndarray:
    lib = _load()
    rp = np.ascontiguousarray(row_ptr, np.int32)
    out = np.empty(rp.shape[0] - 1, np.float32)
    lib.orc_l1_dinv_f32(rp.shape[0] - 1, rp, np.ascontiguousarray(col_idx, np.int32), np.ascontiguousarray(values, np.float32), out)
    return out


def oracle_dadt(coil, transform, didt, nodes_mm) -> np.ndarray:
    lib = _load()
    nodes = np.ascontiguousarray(nodes_mm, np.float64)
    out = np.empty_like(nodes)
    pos = np.ascontiguousarray(coil.positions_m, np.float64)
    lib.orc_dadt(pos, np.ascontiguousarray(coil.moments, np.float64), pos.shape[0],
                 np.ascontiguousarray(transform, np.float64).reshape(16), float(didt), nodes, nodes.shape[0], out)
    return out


def oracle_summary(magnE, vols, bary, tags, region_tag=2) -> np.ndarray:
    lib = _load()
    out = np.empty(SUMMARY_LEN)
    m = np.ascontiguousarray(magnE, np.float32)
    lib.orc_summary(m, np.ascontiguousarray(vols, np.float32), np.ascontiguousarray(bary, np.float64),
                    np.ascontiguousarray(tags, np.int32), m.shape[0], int(region_tag), out)
    return out


def oracle_weighted_quantiles(values, weights, qs) -> np.ndarray:
    lib = _load()
    v = np.ascontiguousarray(values, np.float64)
    q = np.ascontiguousarray(qs, np.float64)
    out = np.empty(q.shape[0])
    lib.orc_weighted_quantiles(v, np.ascontiguousarray(weights, np.float64), v.shape[0], q, q.shape[0], out)
    return out
