"""CPU oracle for the star-join pipeline -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this package, and only as the checker.  The product (practice_b200) never
imports, links or calls it.

``run_plan`` evaluates a plan over host columns with oracle/crystal_oracle.c, a
C restatement of the reference's algorithm (each rule cites the reference file
it follows).  The oracle is pinned against the reference's own known-answer
fixtures (test/nullable_data, test/test_sql_3vl.cpp truth table,
test/test_nullable_semantics.cpp bitmap encodings) committed under
tests/golden/.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libcrystal_oracle.so"


def build() -> Path:
    if not LIB.exists() or LIB.stat().st_mtime < (HERE / "crystal_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "libcrystal_oracle.so"], check=True, capture_output=True)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        P = C.POINTER
        lib.oracle_run.restype = C.c_int
        lib.oracle_run.argtypes = [C.c_char_p, C.c_int, P(C.c_char_p), P(C.c_void_p), P(C.c_void_p), C.c_int,
                                   P(C.c_char_p), P(C.c_longlong), C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                   P(C.c_longlong), C.c_char_p, C.c_int]
        _lib = lib
    return _lib


class OracleResult:
    def __init__(self, words: np.ndarray, validity: np.ndarray, domain_errors: int):
        self.words = words
        self.validity = validity
        self.domain_errors = domain_errors


def run_plan(plan_text: str, columns: dict[str, np.ndarray], validity: dict[str, np.ndarray],
             table_rows: dict[str, int], result_words: int) -> OracleResult:
    lib = _load()
    names = list(columns)
    arrs = [np.ascontiguousarray(columns[n], dtype=np.int32) for n in names]
    vals = [np.ascontiguousarray(validity[n], dtype=np.uint64) if n in validity else None for n in names]
    c_names = (C.c_char_p * len(names))(*[n.encode() for n in names])
    c_data = (C.c_void_p * len(names))(*[a.ctypes.data for a in arrs])
    c_valid = (C.c_void_p * len(names))(*[(v.ctypes.data if v is not None else None) for v in vals])
    tnames = list(table_rows)
    c_tn = (C.c_char_p * len(tnames))(*[t.encode() for t in tnames])
    c_tr = (C.c_longlong * len(tnames))(*[int(table_rows[t]) for t in tnames])
    vwords = (result_words + 63) // 64
    res = np.zeros(max(result_words, 1), dtype=np.uint64)
    val = np.zeros(max(vwords, 1), dtype=np.uint64)
    derr = C.c_longlong(0)
    err = C.create_string_buffer(1024)
    rc = lib.oracle_run(plan_text.encode(), len(names), c_names, c_data, c_valid, len(tnames), c_tn, c_tr,
                        res.ctypes.data, len(res), val.ctypes.data, len(val), C.byref(derr), err, len(err))
    if rc != 0:
        raise RuntimeError(f"oracle: {err.value.decode()}")
    return OracleResult(res[:result_words], val[:vwords], derr.value)
