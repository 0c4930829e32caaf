"""Device primitives of `crystal_sm100.cuh` compiled for the host and checked
against their per-row definitions on the CPU.

`BlockProbeExactBitmap` (exact membership from a shared-memory slot bitmap,
branch-free for in-window keys, outside keys probed through the PHT),
`WarpLoadValidityV` (validity bits of a vector-striped tile, one word load per
lane vector), the PHT build and probe cores and the `BlockPred*` predicates are
plain C++ once `CX_DEVICE` is defined for the host: their source is taken from
the header as it ships, compiled with g++, and compared with the reference
semantics they must keep -- the PHT build and probe of
`include/crystal/join.h:3-250` (a key is a member when the slot `HASH` gives
holds it), `ColumnValidAt` of `include/crystal/load.h:72-76` (bit r of the
uint64 word array) and the set / AND / OR rules of `include/crystal/pred.h`.
"""
from __future__ import annotations

import ctypes
import os
import random
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HEADER = Path(__file__).resolve().parent.parent / "practice_b200" / "csrc" / "crystal_sm100.cuh"
GXX = shutil.which("g++") or "/usr/bin/g++"


def _function(src: str, name: str) -> str:
    """The template header and body of device function `name`."""
    m = re.search(r"(template <[^\n]*>\n)?CX_DEVICE [^\n]*\b" + name + r"\(", src)
    assert m, name
    i = src.index("{", m.end())
    depth = 0
    for j in range(i, len(src)):
        depth += {"{": 1, "}": -1}.get(src[j], 0)
        if depth == 0:
            return src[m.start():j + 1]
    raise AssertionError(f"unbalanced braces in {name}")


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    if not os.path.exists(GXX):
        pytest.skip("needs a host C++ compiler")
    src = HEADER.read_text()
    prelude = src[:src.index("}  // namespace cx_detail") + len("}  // namespace cx_detail")]
    prelude = prelude[prelude.index("#if defined(__CUDACC_RTC__)"):]
    # One host thread: a compare-and-swap is a plain read and conditional write.
    stubs = ("struct int2 { int x, y; };\n"
             "template <class T> static T atomicCAS(T* a, T cmp, T v) { T old = *a; if (old == cmp) *a = v; return old; }\n")
    parts = ["#define CX_DEVICE static inline", prelude, stubs,
             _function(src, "ColumnValidAt"), _function(src, "WarpLoadValidityV"),
             _function(src, "BlockProbeExactBitmap"),
             "namespace cx_detail {", _function(src, "pht_probe"), _function(src, "pht_build"), "}"]
    parts.append("""
template <int IPT>
static void probe_t(int tid, int num_items, const int* items_in, int* flags_io, const unsigned* bitmap,
                    const int* ht, int pair, int len, int key_min) {
  int items[IPT], flags[IPT];
  for (int i = 0; i < IPT; ++i) { items[i] = items_in[i]; flags[i] = flags_io[i]; }
  BlockProbeExactBitmap<int, 32, IPT>(tid, items, flags, bitmap, ht, pair, len, key_min, num_items);
  for (int i = 0; i < IPT; ++i) flags_io[i] = flags[i];
}
extern "C" void probe4(int tid, int n, const int* it, int* fl, const unsigned* bm, const int* ht, int pair, int len,
                       int kmin) { probe_t<4>(tid, n, it, fl, bm, ht, pair, len, kmin); }
extern "C" void probe2(int tid, int n, const int* it, int* fl, const unsigned* bm, const int* ht, int pair, int len,
                       int kmin) { probe_t<2>(tid, n, it, fl, bm, ht, pair, len, kmin); }
template <int IPT>
static void valid_t(const uint64_t* bm, int lane, long long tile_offset, int* out) {
  int v[IPT];
  WarpLoadValidityV<IPT>(bm, lane, tile_offset, v);
  for (int i = 0; i < IPT; ++i) out[i] = v[i];
}
extern "C" void valid1(const uint64_t* bm, int lane, long long off, int* out) { valid_t<1>(bm, lane, off, out); }
extern "C" void valid2(const uint64_t* bm, int lane, long long off, int* out) { valid_t<2>(bm, lane, off, out); }
extern "C" void valid4(const uint64_t* bm, int lane, long long off, int* out) { valid_t<4>(bm, lane, off, out); }
extern "C" void valid8(const uint64_t* bm, int lane, long long off, int* out) { valid_t<8>(bm, lane, off, out); }
template <bool PAIR>
static void build_t(int tid, int n, const int* k_in, const int* v_in, const int* f_in, int* ht, int len, int kmin) {
  int keys[4], vals[4], flags[4];
  for (int i = 0; i < 4; ++i) { keys[i] = k_in[i]; vals[i] = v_in[i]; flags[i] = f_in[i]; }
  cx_detail::pht_build<int, int, 32, 4, PAIR>(tid, keys, vals, flags, ht, len, kmin, n, n != 128);
}
template <bool PAIR>
static void pprobe_t(int tid, int n, const int* k_in, int* f_io, int* res, const int* ht, int len, int kmin) {
  int items[4], flags[4];
  for (int i = 0; i < 4; ++i) { items[i] = k_in[i]; flags[i] = f_io[i]; }
  cx_detail::pht_probe<int, int, 32, 4, PAIR>(tid, items, res, flags, ht, len, kmin, n, n != 128);
  for (int i = 0; i < 4; ++i) f_io[i] = flags[i];
}
extern "C" void build1(int tid, int n, const int* k, const int* v, const int* f, int* ht, int len, int kmin) {
  build_t<false>(tid, n, k, v, f, ht, len, kmin); }
extern "C" void build2(int tid, int n, const int* k, const int* v, const int* f, int* ht, int len, int kmin) {
  build_t<true>(tid, n, k, v, f, ht, len, kmin); }
extern "C" void pprobe1(int tid, int n, const int* k, int* f, int* res, const int* ht, int len, int kmin) {
  pprobe_t<false>(tid, n, k, f, res, ht, len, kmin); }
extern "C" void pprobe2(int tid, int n, const int* k, int* f, int* res, const int* ht, int len, int kmin) {
  pprobe_t<true>(tid, n, k, f, res, ht, len, kmin); }
""")
    d = tmp_path_factory.mktemp("prims")
    cpp, so = d / "prims.cpp", d / "libprims.so"
    cpp.write_text("\n".join(parts) + "\n")
    subprocess.run([GXX, "-O1", "-std=c++17", "-shared", "-fPIC", "-Wno-unknown-pragmas", "-o", str(so), str(cpp)],
                   check=True)
    return ctypes.CDLL(str(so))


def _c_mod(a: int, b: int) -> int:
    """C's % on ints: the remainder takes the dividend's sign."""
    r = abs(a) % abs(b)
    return -r if a < 0 else r


def _slot(key: int, length: int, key_min: int) -> int:
    d = key - key_min
    if 0 <= d < length:
        return d
    h = _c_mod(key - key_min, length)
    return h if 0 <= h < length else -1


def _pht(rng: random.Random, length: int, key_min: int, pair: int):
    """A PHT of `length` slots filled from keys around its window (first key
    into a slot wins), and its exact membership bitmap (bit h set when slot h
    holds key_min + h)."""
    ht = np.zeros(length << pair, dtype=np.int32)
    for _ in range(length):
        k = rng.randint(key_min - 3 * length, key_min + 4 * length)
        h = _slot(k, length, key_min)
        if h >= 0 and ht[h << pair] == 0:
            ht[h << pair] = k
            if pair:
                ht[(h << 1) + 1] = rng.randint(0, 99)
    bm = np.zeros((length + 31) // 32, dtype=np.uint32)
    for h in range(length):
        if ht[h << pair] == key_min + h:
            bm[h >> 5] |= np.uint32(1 << (h & 31))
    return ht, bm


@pytest.mark.parametrize("ipt", [2, 4])
@pytest.mark.parametrize("pair", [0, 1])
def test_exact_bitmap_probe_matches_the_pht_probe(lib, ipt, pair):
    rng = random.Random(1000 * ipt + pair)
    fn = getattr(lib, f"probe{ipt}")
    ip = ctypes.POINTER(ctypes.c_int)
    up = ctypes.POINTER(ctypes.c_uint)
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ip, ip, up, ip, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    for trial in range(300):
        length = rng.choice((1, 7, 32, 100, 1000))
        key_min = rng.choice((1000, 19920101, -500))
        ht, bm = _pht(rng, length, key_min, pair)
        stored = [int(k) for k in ht[::1 << pair] if k != 0]
        tid = rng.randrange(32)
        n = 32 * ipt if rng.random() < 0.5 else rng.randint(0, 32 * ipt)
        items = np.array([rng.choice(stored) if stored and rng.random() < 0.5 else
                          rng.randint(key_min - 5 * length, key_min + 6 * length) for _ in range(ipt)], dtype=np.int32)
        flags = np.array([rng.choice((0, 1, 1, 2)) for _ in range(ipt)], dtype=np.int32)
        want = flags.copy()
        for i in range(ipt):
            if n == 32 * ipt or i * 32 + tid < n:  # live item: the flag keeps only members
                h = _slot(int(items[i]), length, key_min)
                hit = h >= 0 and int(ht[h << pair]) == int(items[i])
                want[i] = int(flags[i] != 0 and hit)
        got = flags.copy()
        fn(tid, n, items.ctypes.data_as(ip), got.ctypes.data_as(ip), bm.ctypes.data_as(up), ht.ctypes.data_as(ip),
           pair, length, key_min)
        assert np.array_equal(got, want), (trial, length, key_min, tid, n, items, flags, got, want)


@pytest.mark.parametrize("ipt", [1, 2, 4, 8])
def test_vector_validity_bits_match_column_valid_at(lib, ipt):
    rng = np.random.default_rng(ipt)
    words = rng.integers(0, 2 ** 64, size=64, dtype=np.uint64)
    fn = getattr(lib, f"valid{ipt}")
    vw = min(ipt, 4)
    out = np.zeros(ipt, dtype=np.int32)
    u64p, ip = ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int)
    fn.argtypes = [u64p, ctypes.c_int, ctypes.c_longlong, ip]
    tiles = (64 * 64) // (32 * ipt)
    for t in range(tiles):
        off = t * 32 * ipt
        for lane in range(32):
            fn(words.ctypes.data_as(u64p), lane, off, out.ctypes.data_as(ip))
            for i in range(ipt):
                r = off + (i // vw) * 32 * vw + lane * vw + i % vw
                assert out[i] == (int(words[r >> 6]) >> (r & 63)) & 1, (t, lane, i)
            fn(None, lane, off, out.ctypes.data_as(ip))  # no bitmap: every row valid
            assert out.tolist() == [1] * ipt


@pytest.mark.parametrize("pair", [0, 1])
def test_pht_build_then_probe_match_the_reference_rules(lib, pair):
    """Build (`BlockBuildSelectivePHT_1/2`: compare-and-swap of the key into
    the slot `HASH` gives; a pair slot takes the payload when the slot was empty
    or already held the key -- the reference writes it unconditionally, which
    differs only when two build keys share a slot, a documented divergence)
    then probe (`BlockProbeAndPHT_1/2`: a member when
    the slot holds the key, the payload read beside it), item by item in the
    same order as a sequential model; keys around and outside the window,
    partial tiles, flags cleared or of any value, odd table addresses (no
    8-byte pair load) and aligned ones."""
    rng = random.Random(77 + pair)
    ip = ctypes.POINTER(ctypes.c_int)
    build = getattr(lib, f"build{pair + 1}")
    probe = getattr(lib, f"pprobe{pair + 1}")
    build.argtypes = [ctypes.c_int, ctypes.c_int, ip, ip, ip, ip, ctypes.c_int, ctypes.c_int]
    probe.argtypes = [ctypes.c_int, ctypes.c_int, ip, ip, ip, ip, ctypes.c_int, ctypes.c_int]
    for trial in range(200):
        length = rng.choice((1, 5, 64, 300))
        key_min = rng.choice((1, 1000, 19920101))
        width = length << pair
        backing = np.zeros(width + 1, dtype=np.int32)
        ht = backing[1:] if trial % 2 else backing[:-1]  # odd trials: table at a 4-byte, not 8-byte, boundary
        model = np.zeros(width, dtype=np.int64)
        for _tile in range(6):
            tid = rng.randrange(32)
            n = 128 if rng.random() < 0.5 else rng.randint(0, 128)
            keys = np.array([rng.randint(key_min - 2 * length, key_min + 3 * length) or 1 for _ in range(4)],
                            dtype=np.int32)
            vals = np.array([rng.randint(1, 50) for _ in range(4)], dtype=np.int32)
            flags = np.array([rng.choice((0, 1, 3)) for _ in range(4)], dtype=np.int32)
            for i in range(4):
                if not (n == 128 or i * 32 + tid < n) or not flags[i]:
                    continue
                h = _slot(int(keys[i]), length, key_min)
                if h < 0:
                    continue
                if pair:
                    prev = model[2 * h]
                    if prev == 0:
                        model[2 * h] = keys[i]
                    if prev == 0 or prev == keys[i]:
                        model[2 * h + 1] = vals[i]
                elif model[h] == 0:
                    model[h] = keys[i]
            build(tid, n, keys.ctypes.data_as(ip), vals.ctypes.data_as(ip), flags.ctypes.data_as(ip),
                  ht.ctypes.data_as(ip), length, key_min)
        assert np.array_equal(ht.astype(np.int64), model), trial
        stored = [int(k) for k in model[::1 << pair] if k != 0]
        for _tile in range(6):
            tid = rng.randrange(32)
            n = 128 if rng.random() < 0.5 else rng.randint(0, 128)
            items = np.array([rng.choice(stored) if stored and rng.random() < 0.6 else
                              rng.randint(key_min - 3 * length, key_min + 4 * length) for _ in range(4)], dtype=np.int32)
            flags = np.array([rng.choice((0, 1, 2)) for _ in range(4)], dtype=np.int32)
            res = np.full(4, -7, dtype=np.int32)
            want_f, want_r = flags.copy(), res.copy()
            for i in range(4):
                if not (n == 128 or i * 32 + tid < n) or not flags[i]:
                    continue
                h = _slot(int(items[i]), length, key_min)
                if h < 0:
                    want_f[i] = 0
                elif pair:
                    if model[2 * h] == items[i]:
                        want_r[i] = model[2 * h + 1]
                    else:
                        want_f[i] = 0
                else:
                    want_f[i] = int(model[h] == items[i])
            probe(tid, n, items.ctypes.data_as(ip), flags.ctypes.data_as(ip), res.ctypes.data_as(ip),
                  ht.ctypes.data_as(ip), length, key_min)
            assert np.array_equal(flags, want_f) and np.array_equal(res, want_r), (trial, items, flags, want_f)


PRED_OPS = {"LT": "<", "GT": ">", "LTE": "<=", "GTE": ">=", "Eq": "==", "NEq": "!="}
# Literal forms (pred.h:153-260): set, AND and OR variants; the OR form of Eq/NEq is spelled BlockPredOr<Op>.
LITERAL_PREDS = [(f"BlockPred{op}", op, "set") for op in PRED_OPS] + \
                [(f"BlockPredA{op}", op, "and") for op in PRED_OPS] + \
                [(f"BlockPredOr{op}" if op in ("Eq", "NEq") else f"BlockPredO{op}", op, "or") for op in PRED_OPS]
COLS_PREDS = [(f"BlockPred{op}_Cols", op, "set") for op in PRED_OPS] + \
             [(f"BlockPredA{op}_Cols", op, "and") for op in PRED_OPS] + \
             [(f"BlockPredOr{op}_Cols", op, "or") for op in PRED_OPS]


@pytest.fixture(scope="module")
def predlib(tmp_path_factory):
    if not os.path.exists(GXX):
        pytest.skip("needs a host C++ compiler")
    src = HEADER.read_text()
    prelude = src[src.index("#if defined(__CUDACC_RTC__)"):src.index("}  // namespace cx_detail") + 26]
    preds = src[src.index("// ------------------------------------------------------------- predicates ---"):
                src.index("// ------------------------------------------------- perfect hash tables (PHT) ---")]
    parts = ["#define CX_DEVICE inline", prelude, preds]  # also marks the functors' members: no `static`
    for name, _, _ in LITERAL_PREDS:
        parts.append(f'extern "C" void lit_{name}(int tid, int n, const int* it, int c, int* fl) {{ int items[4], flags[4];'
                     f" for (int i = 0; i < 4; ++i) {{ items[i] = it[i]; flags[i] = fl[i]; }}"
                     f" {name}<int, 32, 4>(tid, items, flags, c, n); for (int i = 0; i < 4; ++i) fl[i] = flags[i]; }}")
    for name, _, _ in COLS_PREDS:
        parts.append(f'extern "C" void col_{name}(int tid, int n, const int* a, const int* b, int* fl) {{'
                     f" int x[4], y[4], flags[4]; for (int i = 0; i < 4; ++i) {{ x[i] = a[i]; y[i] = b[i]; flags[i] = fl[i]; }}"
                     f" {name}<int, 32, 4>(tid, x, y, flags, n); for (int i = 0; i < 4; ++i) fl[i] = flags[i]; }}")
    d = tmp_path_factory.mktemp("preds")
    cpp, so = d / "preds.cpp", d / "libpreds.so"
    cpp.write_text("\n".join(parts) + "\n")
    subprocess.run([GXX, "-O1", "-std=c++17", "-shared", "-fPIC", "-Wno-unknown-pragmas", "-o", str(so), str(cpp)],
                   check=True)
    return ctypes.CDLL(str(so))


def _cmp(op: str, x: int, y: int) -> bool:
    return {"LT": x < y, "GT": x > y, "LTE": x <= y, "GTE": x >= y, "Eq": x == y, "NEq": x != y}[op]


def _combine(mode: str, flag: int, p: bool) -> int:
    return int(p) if mode == "set" else int(bool(flag) and p) if mode == "and" else int(bool(flag) or p)


@pytest.mark.parametrize("cols", [False, True])
def test_block_predicates_follow_the_reference_combine_rules(predlib, cols):
    """`BlockPred*` set the flag, `BlockPredA*` AND into it, `BlockPredO*` /
    `BlockPredOr*` OR into it, for items inside the tile (a full tile: all;
    else item i of thread tid when i * 32 + tid < num_items); other items keep
    their flag.  Literal and column-vs-column forms (pred.h:153-445)."""
    rng = random.Random(5 + cols)
    ip = ctypes.POINTER(ctypes.c_int)
    for name, op, mode in (COLS_PREDS if cols else LITERAL_PREDS):
        fn = getattr(predlib, ("col_" if cols else "lit_") + name)
        fn.argtypes = [ctypes.c_int, ctypes.c_int, ip, ip, ip] if cols else [ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, ip]
        for _ in range(100):
            tid = rng.randrange(32)
            n = 128 if rng.random() < 0.4 else rng.randint(0, 128)
            a = np.array([rng.randint(-3, 3) for _ in range(4)], dtype=np.int32)
            b = np.array([rng.randint(-3, 3) for _ in range(4)], dtype=np.int32)
            c = rng.randint(-3, 3)
            flags = np.array([rng.choice((0, 1, 2)) for _ in range(4)], dtype=np.int32)
            want = flags.copy()
            for i in range(4):
                if n == 128 or i * 32 + tid < n:
                    want[i] = _combine(mode, int(flags[i]), _cmp(op, int(a[i]), int(b[i]) if cols else c))
            if cols:
                fn(tid, n, a.ctypes.data_as(ip), b.ctypes.data_as(ip), flags.ctypes.data_as(ip))
            else:
                fn(tid, n, a.ctypes.data_as(ip), c, flags.ctypes.data_as(ip))
            assert np.array_equal(flags, want), (name, tid, n, a, b, c, flags, want)
