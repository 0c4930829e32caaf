"""ctypes binding of libcrystal_b200.so (include/crystal_b200.h).

The library is the product: if it is missing, importing this module raises
instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcrystal_b200.so"

CX_OK = 0
ERRORS = {
    -1: "CX_E_INVALID", -2: "CX_E_COMPILE", -3: "CX_E_CUDA", -4: "CX_E_MISSING",
    -5: "CX_E_CAPACITY", -6: "CX_E_KERNEL", -7: "CX_E_NO_DEVICE", -8: "CX_E_REJECTED",
}

# Every symbol include/crystal_b200.h declares (checked by the CPU tests).
EXPORTS = [
    "cx_abi_version", "cx_last_error", "cx_tuning_default", "cx_codegen", "cx_translate_visitor", "cx_compile",
    "cx_module_release", "cx_module_result_info", "cx_ctx_create", "cx_ctx_destroy",
    "cx_ctx_set_buffer", "cx_ctx_set_null_bitmap", "cx_ctx_set_table_rows", "cx_ctx_set_result",
    "cx_ctx_set_scratch", "cx_module_scratch_bytes", "cx_ctx_set_sm_count", "cx_execute",
    "cx_execute_params", "cx_ctx_sync", "cx_ctx_timing", "cx_ctx_kernel_error", "cx_compact_sparse", "cx_compact_sparse_noalloc",
    "cx_gen_uniform", "cx_gen_datekey", "cx_gen_validity", "cx_plan_literals", "cx_shared_codegen",
    "cx_shared_execute", "cx_shared_execute_rows", "cx_ctx_set_column_range", "cx_ctx_set_graph_replay",
    "cx_server_config_default", "cx_server_create", "cx_server_prepare", "cx_server_prepare_tuned",
    "cx_server_submit", "cx_server_wait",
    "cx_server_fetch", "cx_server_release", "cx_server_get_stats", "cx_server_destroy", "cx_finalize",
]


class CxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Tuning(C.Structure):
    _fields_ = [("block_threads", C.c_int), ("items_per_thread", C.c_int), ("stages", C.c_int),
                ("ctas_per_sm", C.c_int), ("group_placement", C.c_int), ("smem_group_budget", C.c_int),
                ("bitmap_budget", C.c_int), ("group_merge", C.c_int), ("producer_warps", C.c_int),
                ("parametric", C.c_int), ("prefetch", C.c_int), ("wait_limit_us", C.c_int),
                ("debug_stall", C.c_int), ("compact", C.c_int), ("table_budget", C.c_int), ("cube", C.c_int)]


class ResultInfo(C.Structure):
    _fields_ = [("groups", C.c_uint64), ("storage_ts", C.c_uint32), ("visible_ts", C.c_uint32),
                ("result_words", C.c_uint64), ("validity_words", C.c_uint64), ("final_words", C.c_uint64),
                ("sparse", C.c_int), ("finalized", C.c_int)]


class SharedQuery(C.Structure):
    _fields_ = [("shape", C.c_int), ("param_off", C.c_int), ("result", C.c_void_p), ("result_words", C.c_uint64),
                ("validity", C.c_void_p), ("validity_words", C.c_uint64)]


class ResultLayout(C.Structure):
    _fields_ = [("groups", C.c_uint64), ("tuple_size", C.c_uint32), ("columns", C.c_uint32), ("sparse", C.c_int),
                ("scalar", C.c_int), ("column_type", C.POINTER(C.c_uint8)), ("column_nullable", C.POINTER(C.c_uint8))]


class SortKey(C.Structure):
    _fields_ = [("column", C.c_int), ("descending", C.c_int)]


class ServerConfig(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("max_batch", C.c_int), ("slots", C.c_int), ("plain_only", C.c_int),
                ("min_shared_batch", C.c_int), ("shared_tuning", Tuning), ("chunk_rows", C.c_uint64),
                ("cube_bytes", C.c_uint64)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("kernel_error", C.c_uint32), ("words", C.c_uint64),
                ("validity_words", C.c_uint64), ("queue_ms", C.c_double), ("latency_ms", C.c_double),
                ("batch_size", C.c_int), ("shared", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("rejected", C.c_uint64),
                ("launches", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("mean_batch", C.c_double), ("queries_per_s", C.c_double), ("budget_bytes", C.c_uint64),
                ("peak_reserved_bytes", C.c_uint64)]


class Timing(C.Structure):
    _fields_ = [("build_ms", C.c_float), ("scan_ms", C.c_float), ("post_ms", C.c_float),
                ("total_ms", C.c_float), ("scan_grid", C.c_int), ("gpu_launches", C.c_int), ("graph", C.c_int),
                ("mode", C.c_int)]


# CX_ABI_VERSION of include/crystal_b200.h that the structures above mirror.
ABI_VERSION = 1


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `python -m practice_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    vp, u64, i64, u32, sz = C.c_void_p, C.c_uint64, C.c_int64, C.c_uint32, C.c_size_t
    sig = {
        "cx_abi_version": (C.c_int, []),
        "cx_last_error": (C.c_char_p, []),
        "cx_tuning_default": (None, [C.POINTER(Tuning)]),
        "cx_codegen": (C.c_int, [C.c_char_p, sz, C.POINTER(Tuning), C.c_char_p, sz, C.POINTER(sz)]),
        "cx_translate_visitor": (C.c_int, [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
        "cx_compile": (C.c_int, [C.c_char_p, sz, C.c_char_p, C.POINTER(vp), C.c_char_p, sz]),
        "cx_module_release": (C.c_int, [vp]),
        "cx_module_result_info": (C.c_int, [vp, C.POINTER(ResultInfo)]),
        "cx_ctx_create": (vp, []),
        "cx_ctx_destroy": (None, [vp]),
        "cx_ctx_set_buffer": (C.c_int, [vp, C.c_char_p, vp, u64]),
        "cx_ctx_set_null_bitmap": (C.c_int, [vp, C.c_char_p, vp, u64]),
        "cx_ctx_set_table_rows": (C.c_int, [vp, C.c_char_p, u64]),
        "cx_ctx_set_result": (C.c_int, [vp, vp, u64, vp, u64]),
        "cx_ctx_set_scratch": (C.c_int, [vp, vp, u64]),
        "cx_module_scratch_bytes": (C.c_int, [vp, vp, C.POINTER(u64)]),
        "cx_ctx_set_sm_count": (C.c_int, [vp, C.c_int]),
        "cx_ctx_set_column_range": (C.c_int, [vp, C.c_char_p, i64, i64]),
        "cx_ctx_set_graph_replay": (C.c_int, [vp, C.c_int]),
        "cx_server_config_default": (None, [C.POINTER(ServerConfig)]),
        "cx_server_create": (C.c_int, [vp, C.POINTER(ServerConfig), C.POINTER(vp)]),
        "cx_server_prepare": (C.c_int, [vp, C.c_char_p, sz]),
        "cx_server_prepare_tuned": (C.c_int, [vp, C.c_char_p, sz, C.POINTER(Tuning)]),
        "cx_server_submit": (C.c_int, [vp, C.c_char_p, sz, C.POINTER(u64)]),
        "cx_server_wait": (C.c_int, [vp, u64, C.c_int, C.POINTER(RequestInfo)]),
        "cx_server_fetch": (C.c_int, [vp, u64, vp, u64, vp, u64]),
        "cx_server_release": (C.c_int, [vp, u64]),
        "cx_server_get_stats": (C.c_int, [vp, C.c_int, C.POINTER(ServerStats)]),
        "cx_server_destroy": (C.c_int, [vp]),
        "cx_finalize": (C.c_int, [vp, vp, C.POINTER(ResultLayout), C.POINTER(SortKey), C.c_int, u64, vp, vp, u64,
                                  C.POINTER(u64), vp]),
        "cx_execute": (C.c_int, [vp, vp, vp]),
        "cx_execute_params": (C.c_int, [vp, vp, C.POINTER(C.c_int32), C.c_int, vp]),
        "cx_ctx_sync": (C.c_int, [vp]),
        "cx_ctx_timing": (C.c_int, [vp, C.POINTER(Timing)]),
        "cx_ctx_kernel_error": (C.c_int, [vp, C.POINTER(u32)]),
        "cx_compact_sparse": (C.c_int, [vp, u64, u32, vp, vp, vp]),
        "cx_compact_sparse_noalloc": (C.c_int, [vp, u64, u32, vp, vp, vp]),
        "cx_gen_uniform": (C.c_int, [u64, u64, i64, i64, u64, u64, vp, vp]),
        "cx_gen_datekey": (C.c_int, [u64, u64, u32, u64, u64, vp, vp]),
        "cx_gen_validity": (C.c_int, [u64, u64, u64, u32, vp, vp]),
        "cx_plan_literals": (C.c_int, [C.c_char_p, sz, C.POINTER(i64), C.c_int, C.POINTER(C.c_int)]),
        "cx_shared_codegen": (C.c_int, [C.POINTER(C.c_char_p), C.POINTER(sz), C.c_int, C.POINTER(Tuning), C.c_char_p,
                                        sz, C.POINTER(sz)]),
        "cx_shared_execute": (C.c_int, [vp, vp, C.POINTER(SharedQuery), C.c_int, C.POINTER(C.c_int32), C.c_int, vp]),
        "cx_shared_execute_rows": (C.c_int, [vp, vp, C.POINTER(SharedQuery), C.c_int, C.POINTER(C.c_int32), C.c_int,
                                             u64, u64, C.POINTER(C.c_uint8), vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.cx_abi_version() != ABI_VERSION:
        raise ImportError(f"{LIB_PATH} has C ABI version {lib.cx_abi_version()}, these bindings expect "
                          f"{ABI_VERSION}; rebuild with `python -m practice_b200.build`")
    return lib


lib = _load()


def check(rc: int, what: str = "") -> None:
    if rc != CX_OK:
        msg = lib.cx_last_error().decode(errors="replace")
        raise CxError(rc, f"{what}: {msg}" if what else msg)


def default_tuning() -> Tuning:
    t = Tuning()
    lib.cx_tuning_default(C.byref(t))
    return t


def codegen(plan_text: str, tuning: Tuning | None = None) -> str:
    raw = plan_text.encode()
    n = C.c_size_t(0)
    tp = C.byref(tuning) if tuning is not None else None
    check(lib.cx_codegen(raw, len(raw), tp, None, 0, C.byref(n)), "cx_codegen")
    buf = C.create_string_buffer(n.value + 1)
    check(lib.cx_codegen(raw, len(raw), tp, buf, n.value + 1, C.byref(n)), "cx_codegen")
    return buf.value.decode()


def translate_visitor(source: str) -> str:
    """The CUDA program cx_compile makes of a program emitted by the reference's
    code generator (its kernel bodies under this library's launch skeleton)."""
    n = C.c_size_t(0)
    src = source.encode()
    check(lib.cx_translate_visitor(src, len(src), None, 0, C.byref(n)), "cx_translate_visitor")
    buf = C.create_string_buffer(n.value + 1)
    check(lib.cx_translate_visitor(src, len(src), buf, len(buf), C.byref(n)), "cx_translate_visitor")
    return buf.value.decode()


def plan_literals(plan_text: str) -> list[int]:
    raw = plan_text.encode()
    n = C.c_int(0)
    check(lib.cx_plan_literals(raw, len(raw), None, 0, C.byref(n)), "cx_plan_literals")
    out = (C.c_int64 * max(n.value, 1))()
    check(lib.cx_plan_literals(raw, len(raw), out, n.value, C.byref(n)), "cx_plan_literals")
    return list(out[: n.value])


def shared_codegen(plan_texts: list[str], tuning: Tuning | None = None) -> str:
    raws = [t.encode() for t in plan_texts]
    arr = (C.c_char_p * len(raws))(*raws)
    lens = (C.c_size_t * len(raws))(*[len(r) for r in raws])
    n = C.c_size_t(0)
    tp = C.byref(tuning) if tuning is not None else None
    check(lib.cx_shared_codegen(arr, lens, len(raws), tp, None, 0, C.byref(n)), "cx_shared_codegen")
    buf = C.create_string_buffer(n.value + 1)
    check(lib.cx_shared_codegen(arr, lens, len(raws), tp, buf, n.value + 1, C.byref(n)), "cx_shared_codegen")
    return buf.value.decode()


class Module:
    """A compiled query (cx_module*)."""

    def __init__(self, source: str, key: str | None = None):
        raw = source.encode()
        handle = C.c_void_p()
        log = C.create_string_buffer(1 << 16)
        rc = lib.cx_compile(raw, len(raw), key.encode() if key else None, C.byref(handle), log, len(log))
        if rc != CX_OK:
            raise CxError(rc, lib.cx_last_error().decode(errors="replace"))
        self.handle = handle
        self.source = source
        self.log = log.value.decode(errors="replace")
        info = ResultInfo()
        check(lib.cx_module_result_info(self.handle, C.byref(info)), "cx_module_result_info")
        self.info = info
        sb = C.c_uint64()
        check(lib.cx_module_scratch_bytes(self.handle, None, C.byref(sb)), "cx_module_scratch_bytes")
        self.scratch_bytes = sb.value

    def close(self) -> None:
        if self.handle:
            lib.cx_module_release(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


class ExecCtx:
    """An execution context (cx_exec_ctx*): named device buffers and scratch."""

    def __init__(self):
        self.handle = lib.cx_ctx_create()
        if not self.handle:
            raise MemoryError("cx_ctx_create failed")

    def set_buffer(self, name: str, ptr: int, elems: int) -> None:
        check(lib.cx_ctx_set_buffer(self.handle, name.encode(), ptr, elems), "cx_ctx_set_buffer")

    def set_null_bitmap(self, name: str, ptr: int, words: int) -> None:
        check(lib.cx_ctx_set_null_bitmap(self.handle, name.encode(), ptr, words), "cx_ctx_set_null_bitmap")

    def set_rows(self, table: str, rows: int) -> None:
        check(lib.cx_ctx_set_table_rows(self.handle, table.encode(), rows), "cx_ctx_set_table_rows")

    def set_graph_replay(self, enable: bool) -> None:
        check(lib.cx_ctx_set_graph_replay(self.handle, int(enable)), "cx_ctx_set_graph_replay")

    def set_column_range(self, name: str, lo: int, hi: int) -> None:
        check(lib.cx_ctx_set_column_range(self.handle, name.encode(), lo, hi), "cx_ctx_set_column_range")

    def set_result(self, res_ptr: int, res_words: int, val_ptr: int, val_words: int) -> None:
        check(lib.cx_ctx_set_result(self.handle, res_ptr, res_words, val_ptr, val_words), "cx_ctx_set_result")

    def set_scratch(self, ptr: int | None, nbytes: int) -> None:
        check(lib.cx_ctx_set_scratch(self.handle, ptr, nbytes), "cx_ctx_set_scratch")

    def execute(self, module: Module, stream: int = 0, params=None) -> None:
        if params is None:
            check(lib.cx_execute(module.handle, self.handle, stream or None), "cx_execute")
            return
        pa = (C.c_int32 * max(len(params), 1))(*params)
        check(lib.cx_execute_params(module.handle, self.handle, pa, len(params), stream or None), "cx_execute_params")

    def shared_execute(self, module: Module, queries, params, stream: int = 0) -> None:
        nq = len(queries)
        qa = (SharedQuery * max(nq, 1))(*queries)
        pa = (C.c_int32 * max(len(params), 1))(*params)
        check(lib.cx_shared_execute(module.handle, self.handle, qa, nq, pa, len(params), stream or None),
              "cx_shared_execute")

    def shared_execute_rows(self, module: Module, queries, params, row0: int, nrows: int, keep=None,
                            stream: int = 0) -> None:
        """The batch over fact rows [row0, row0 + nrows); queries whose `keep`
        entry is true add to the result earlier row ranges left."""
        nq = len(queries)
        qa = (SharedQuery * max(nq, 1))(*queries)
        pa = (C.c_int32 * max(len(params), 1))(*params)
        ka = (C.c_uint8 * max(nq, 1))(*[1 if k else 0 for k in keep]) if keep is not None else None
        check(lib.cx_shared_execute_rows(module.handle, self.handle, qa, nq, pa, len(params), row0, nrows, ka,
                                         stream or None), "cx_shared_execute_rows")

    def sync(self) -> None:
        check(lib.cx_ctx_sync(self.handle), "cx_ctx_sync")

    def timing(self) -> Timing:
        t = Timing()
        check(lib.cx_ctx_timing(self.handle, C.byref(t)), "cx_ctx_timing")
        return t

    def kernel_error(self) -> int:
        v = C.c_uint32()
        check(lib.cx_ctx_kernel_error(self.handle, C.byref(v)))
        return v.value

    def close(self) -> None:
        if self.handle:
            lib.cx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def server_config(**kw) -> ServerConfig:
    cfg = ServerConfig()
    lib.cx_server_config_default(C.byref(cfg))
    for k, v in kw.items():
        if k == "shared_tuning":
            cfg.shared_tuning = v
        else:
            setattr(cfg, k, v)
    return cfg


class Server:
    """The request loop (cx_server_*): submit plans as they arrive, wait for
    and fetch each result; queries are admitted against the HBM budget and
    fused into shared-scan launches by the library's scheduler thread."""

    def __init__(self, tables: "ExecCtx", cfg: ServerConfig | None = None):
        self.handle = C.c_void_p()
        check(lib.cx_server_create(tables.handle, C.byref(cfg) if cfg is not None else None, C.byref(self.handle)),
              "cx_server_create")

    def prepare(self, plan_text: str, plain_tuning: Tuning | None = None) -> None:
        raw = plan_text.encode()
        if plain_tuning is None:
            check(lib.cx_server_prepare(self.handle, raw, len(raw)), "cx_server_prepare")
        else:
            check(lib.cx_server_prepare_tuned(self.handle, raw, len(raw), C.byref(plain_tuning)), "cx_server_prepare_tuned")

    def submit(self, plan_text: str) -> int:
        raw = plan_text.encode()
        rid = C.c_uint64()
        check(lib.cx_server_submit(self.handle, raw, len(raw), C.byref(rid)), "cx_server_submit")
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1) -> RequestInfo:
        info = RequestInfo()
        rc = lib.cx_server_wait(self.handle, rid, timeout_ms, C.byref(info))
        if rc not in (CX_OK, -6):
            check(rc, "cx_server_wait")
        return info

    def fetch(self, rid: int, info: RequestInfo):
        import numpy as np

        w = np.zeros(max(int(info.words), 1), dtype=np.uint64)
        v = np.zeros(max(int(info.validity_words), 1), dtype=np.uint64)
        check(lib.cx_server_fetch(self.handle, rid, w.ctypes.data, w.size, v.ctypes.data, v.size), "cx_server_fetch")
        return w[: int(info.words)], v[: int(info.validity_words)]

    def release(self, rid: int) -> None:
        check(lib.cx_server_release(self.handle, rid), "cx_server_release")

    def stats(self, reset: bool = False) -> ServerStats:
        st = ServerStats()
        check(lib.cx_server_get_stats(self.handle, int(reset), C.byref(st)), "cx_server_get_stats")
        return st

    def close(self) -> None:
        if self.handle:
            lib.cx_server_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


COL_INT64, COL_UINT64, COL_FLOAT64 = 0, 1, 2


def finalize(result_ptr: int, validity_ptr: int, groups: int, tuple_size: int, types: list[int],
             nullable: list[bool], sparse: bool, scalar: bool, keys: list[tuple[int, bool]], limit: int | None,
             cols_ptr: int, cvalid_ptr: int, row_cap: int, stream: int = 0) -> int:
    """cx_finalize: result rows written column by column on the device; returns the row count."""
    n = len(types)
    ta = (C.c_uint8 * n)(*types)
    na = (C.c_uint8 * n)(*[int(x) for x in nullable])
    lay = ResultLayout(groups, tuple_size, n, int(sparse), int(scalar), ta, na)
    ka = (SortKey * max(len(keys), 1))(*[SortKey(c, int(d)) for c, d in keys])
    rows = C.c_uint64()
    lim = (1 << 64) - 1 if limit is None else limit
    check(lib.cx_finalize(result_ptr, validity_ptr or None, C.byref(lay), ka, len(keys), lim, cols_ptr, cvalid_ptr,
                          row_cap, C.byref(rows), stream or None), "cx_finalize")
    return rows.value
