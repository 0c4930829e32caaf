"""CPU tests of the product library: it loads without a GPU, exports every
symbol include/crystal_b200.h declares, generates CUDA for every workload plan
and compiles it with NVRTC for sm_100a (NVRTC needs no device), and rejects bad
input with status codes instead of exceptions."""
import random
import re
from pathlib import Path

import pytest

from practice_b200 import _lib, datagen, queries
from practice_b200.plan import PlanBuilder, Table, col, lit, star

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "crystal_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cx_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(_lib.lib, s), s
    assert sorted(_lib.EXPORTS) == syms
    assert _lib.lib.cx_abi_version() == 1


def all_plans():
    rng = random.Random(3)
    plans = {"ssb_q11": queries.ssb_q11(), "ssb_q31": queries.ssb_q31(), "ssb_q31_nullable": queries.ssb_q31_nullable()}
    for t in range(4):
        plans[f"T{t}"] = queries.template(t, rng)
    for k, p in queries.kat_plans().items():
        plans["kat_" + k] = p
    for name in ("or_join_year", "or_join_then_filter", "mht_year_tier", "mht_then_supplier", "mht_brand"):
        plans[name] = getattr(queries, name)()
    return plans


@pytest.mark.parametrize("name", list(all_plans()))
def test_generated_source_compiles_for_sm100a(name):
    plan = all_plans()[name]
    src = _lib.codegen(plan.text())
    assert src.startswith("/*@cx-launch")
    m = _lib.Module(src, key="cpu_" + name)
    assert m.info.result_words == plan.group_slots * plan.storage_ts
    assert m.info.sparse == int(plan.sparse)
    if plan.steps and any(k == "join" for k, _ in plan.steps):
        assert any(k in src for k in ("BlockProbeAndPHT", "BlockProbeExactBitmap", "BlockProbeExactTable", "ProbeMultiHT",
                                     "pht_slot"))
        assert "build_hashtable_" in src or "mht_count_" in src
    if any(k == "join" and s.multi for k, s in plan.steps):
        for kern in ("mht_count_", "mht_blocksum_", "mht_blockscan_", "mht_offsets_", "mht_write_"):
            assert kern in src
    assert "cp.async.bulk" not in src  # staging goes through the header helper
    assert "WarpLoadTileV" in src      # default: unstaged vector loads
    t = _lib.default_tuning()
    t.block_threads, t.stages = 256, 3
    assert "cx::bulk_g2s" in _lib.codegen(plan.text(), t)


@pytest.mark.parametrize("bt,ipt,stages,place", [(128, 4, 4, 0), (256, 8, 2, 0), (512, 2, 3, 2), (256, 4, 0, 1),
                                                 (1024, 1, 2, 0)])
def test_tuning_space_compiles(bt, ipt, stages, place):
    t = _lib.default_tuning()
    t.block_threads, t.items_per_thread, t.stages, t.group_placement = bt, ipt, stages, place
    for name in ("ssb_q31", "ssb_q31_nullable"):
        plan = all_plans()[name]
        _lib.Module(_lib.codegen(plan.text(), t), key=f"tune_{name}_{bt}_{ipt}_{stages}_{place}")


@pytest.mark.parametrize("prefetch,place,merge", [(0, 4, 0), (1, 3, 0), (2, 0, 0), (1, 0, 1), (1, 2, 2), (1, 1, 1),
                                                   (3, 0, 0)])
def test_launch_knobs_compile(prefetch, place, merge):
    """Unstaged loads (where first used / vector loads at the tile start / one
    tile ahead / an L2 prefetch of the next tile), per-thread shared-memory and register group slots, warp-merged
    and per-lane group updates, including the expanding joins' uniform loop."""
    t = _lib.default_tuning()
    t.prefetch, t.group_placement, t.group_merge = prefetch, place, merge
    plans = all_plans()
    for name in ("T1", "T2", "ssb_q31_nullable", "or_join_then_filter", "mht_year_tier"):
        src = _lib.codegen(plans[name].text(), t)
        if prefetch == 0:
            assert "WarpLoadTileV" not in src
        if prefetch == 3 and name in ("T1", "T2"):
            assert "l2_prefetch_bulk" in src
        if place == 4 and name == "T1":
            assert "s_lacc" in src
        _lib.Module(src, key=f"knobs_{name}_{prefetch}_{place}_{merge}")


def test_reference_style_primitive_calls_compile_against_header():
    """Lines in the shape the reference visitor emits (visitor.cpp:4233-4288,
    1838-1880, 4640-4660) compile against crystal_sm100.cuh unchanged."""
    src = r'''/*@cx-launch
v 1
@*/
#include "cx_args.h"
#include "crystal_sm100.cuh"
extern "C" __global__ void ref_style(int* d_lo_quantity, int* d_lo_orderdate, int* d_d_hash_table,
                                     unsigned long long* d_result, uint64_t* n_lo_quantity, int n) {
  constexpr int BLOCK_THREADS = 128, ITEMS_PER_THREAD = 4, TILE_SIZE = 512;
  int tid = threadIdx.x;
  int tile_offset = blockIdx.x * TILE_SIZE;
  int num_tile_items = (blockIdx.x == gridDim.x - 1) ? n - tile_offset : TILE_SIZE;
  int items[ITEMS_PER_THREAD]; int flags[ITEMS_PER_THREAD]; int items2[ITEMS_PER_THREAD];
  int items_valid[ITEMS_PER_THREAD]; int d_year[ITEMS_PER_THREAD];
  InitFlags<BLOCK_THREADS, ITEMS_PER_THREAD>(flags);
  BlockLoad<int, BLOCK_THREADS, ITEMS_PER_THREAD>(d_lo_quantity + tile_offset, tid, tile_offset, items, num_tile_items);
  BlockLoadValidity<BLOCK_THREADS, ITEMS_PER_THREAD>(n_lo_quantity, tid, tile_offset, items_valid, num_tile_items);
  BlockPredAGTE<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, 2, num_tile_items);
  BlockPredOrEq<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, 7, num_tile_items);
  BlockApplyValidityAnd<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, flags, items_valid, num_tile_items);
  BlockLoad<int, BLOCK_THREADS, ITEMS_PER_THREAD>(d_lo_orderdate + tile_offset, tid, tile_offset, items2, num_tile_items);
  BlockProbeAndPHT_2<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items2, d_year, flags, d_d_hash_table, 61131, 19920101, num_tile_items);
  BlockBuildSelectivePHT_1<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, d_d_hash_table, 61131, 19920101, num_tile_items);
  BlockPredALT_Cols<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, items2, flags, num_tile_items);
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (flags[i] && (tid + BLOCK_THREADS * i < num_tile_items)) {
      int hash = (d_year[i] - 1992) % 7;
      d_result[hash * 2] = static_cast<unsigned long long>(d_year[i]);
      db::atomic_add_ull(d_result[hash * 2 + 1], (unsigned long long)items[i] * items2[i]);
      if (db::safe_lt(items[i], db::safe_mul(items2[i], 3))) db::atomic_min_ull(d_result[0], 1ULL);
    }
  }
}
'''
    _lib.Module(src, key="ref_style_snippet")


def test_bad_plans_return_invalid_status():
    with pytest.raises(_lib.CxError) as e:
        _lib.codegen("(query (table T fact (cols qty)) (filter (col nope)) (aggregate (count (star))))")
    assert e.value.code == -1 and "nope" in str(e.value)
    with pytest.raises(_lib.CxError):
        _lib.codegen("(query (table T fact (cols qty)))")  # no aggregate
    with pytest.raises(_lib.CxError):
        _lib.codegen("(query (table T fact (cols qty)) (aggregate (group (add (col qty) (int 1)) (min 0) (card 2)) "
                     "(count (star))))")
    with pytest.raises(_lib.CxError) as e:
        _lib.Module("__global__ void k() {}")
    assert e.value.code == -1


def test_bad_or_and_multi_value_joins_are_rejected():
    base = ("(query (table F fact (cols f1 f2 f3 val)) (table D (cols dkey pay1 pay2)) {join} "
            "(aggregate (sum (col val))))")
    ok = "(join D (pk dkey) (fk f1 f2) (len 10) (keymin 0) (multi 1) (payload pay1 pay2))"
    _lib.codegen(base.format(join=ok))
    bad = {
        "(join D (pk dkey) (fk f1 f1) (len 10) (keymin 0))": "listed twice",
        "(join D (pk dkey) (fk f1 f2 f3 f1 f2) (len 10) (keymin 0))": "at most 4",
        "(join D (pk dkey) (fk f1) (len 10) (keymin 0) (payload pay1 pay2))": "one payload",
        "(join D (pk dkey) (fk f1) (len 10) (keymin 0) (multi 1) (payload pay1 pay1))": "listed twice",
        "(join D (pk dkey) (fk f1) (len 10) (keymin 0) (multi 1) (payload zz))": "not a column",
    }
    for join, msg in bad.items():
        with pytest.raises(_lib.CxError) as e:
            _lib.codegen(base.format(join=join))
        assert e.value.code == -1 and msg in str(e.value), (join, str(e.value))


def test_compile_errors_come_back_with_the_nvrtc_log():
    with pytest.raises(_lib.CxError) as e:
        _lib.Module("/*@cx-launch\nv 1\n@*/\n__global__ void k() { this is not cuda; }", key="broken")
    assert e.value.code == -2 and "error" in str(e.value)


def test_module_cache_reuses_compiled_source():
    plan = all_plans()["kat_q3"]
    src = _lib.codegen(plan.text())
    a = _lib.Module(src, key="cache_probe")
    b = _lib.Module(src, key="cache_probe")
    assert a.handle.value == b.handle.value


def test_execute_without_bound_buffers_reports_missing():
    plan = all_plans()["kat_q3"]
    m = _lib.Module(_lib.codegen(plan.text()), key="missing_probe")
    ctx = _lib.ExecCtx()
    with pytest.raises(_lib.CxError) as e:
        ctx.execute(m)
    assert e.value.code == -4  # rows of NULLABLE_NUMBERS not set: fails before touching a GPU
    ctx.set_rows("NULLABLE_NUMBERS", 12)
    with pytest.raises(_lib.CxError) as e:
        ctx.execute(m)
    assert e.value.code == -4 and "d_val" in str(e.value)


def test_scratch_and_result_shapes():
    plan = all_plans()["ssb_q31_nullable"]
    m = _lib.Module(_lib.codegen(plan.text()), key="shape_probe")
    assert m.info.groups == 251 * 7
    assert m.info.storage_ts == 5 and m.info.visible_ts == 5
    # three hash tables of 2*len ints each plus the payload-validity bits of c_city
    assert m.scratch_bytes >= 4 * 2 * (300_000 + 20_000 + 61131)


def test_plan_text_is_deterministic():
    assert queries.ssb_q31().text() == queries.ssb_q31().text()
    t = {"T": Table("T", ["a"], 1, fact=True)}
    p = PlanBuilder(t, "T").filter(col("a").gt(3)).aggregate([], [("count", star())])
    assert "(filter (gt (col a) (int 3)))" in p.text()


def test_shared_program_for_the_four_templates_compiles():
    rng = random.Random(11)
    plans = [queries.template(t, rng) for t in range(4)]
    src = _lib.shared_codegen([p.text() for p in plans])
    assert "SharedScan_LINEORDER" in src and "index_customer" in src
    m = _lib.Module(src, key="cpu_shared_templates")
    assert m.info.result_words >= 0
    # literals come back in the order that numbers the shape's parameters
    assert _lib.plan_literals(plans[1].text())[0] == plans[1].steps[0][1].kids[1].val


def test_shared_program_carries_the_cube_path_when_shapes_allow():
    rng = random.Random(13)
    texts = [queries.template(t, rng).text() for t in range(4)]
    src = _lib.shared_codegen(texts)
    assert "CubeScan_LINEORDER" in src and "cube_answer" in src and "cube_index_part" in src
    launch = src.split("@*/")[0]
    # quantity, discount, c_region, s_region, d_year, c_nation, p_category, p_brand1
    assert "\ncube 8\n" in launch
    from practice_b200.engine import SHARED_DEFAULT, make_tuning
    assert _lib.default_tuning().cube == 4
    t = make_tuning(**{**SHARED_DEFAULT, "cube": 0})
    assert "CubeScan" not in _lib.shared_codegen(texts, t) and "SharedScan_LINEORDER" in _lib.shared_codegen(texts, t)
    for ipt in (1, 2):
        t.cube = ipt
        m = _lib.Module(_lib.shared_codegen(texts, t), key=f"cpu_cube_{ipt}")
        assert m.info.result_words >= 0
    # An aggregate that reads a literal cannot be summed once for every query of its shape.
    tables = datagen.ssb_tables(1000, queries.BATCH_COLS)
    b = PlanBuilder(tables, "LINEORDER", name="L")
    b.filter(col("lo_quantity").lt(10))
    lit_agg = b.aggregate([], [("sum", col("lo_revenue") * lit(3))]).text()
    assert "CubeScan" not in _lib.shared_codegen([lit_agg] + texts)


def test_shared_program_rejects_unshareable_shapes():
    with pytest.raises(_lib.CxError):
        _lib.shared_codegen([queries.ssb_q31_nullable(1000).text()])  # nullable columns
    with pytest.raises(_lib.CxError):
        _lib.shared_codegen([queries.kat_plans()["q1"].text()])  # AVG


def test_shared_execute_validates_before_touching_the_gpu():
    rng = random.Random(12)
    p = queries.template(2, rng)
    m = _lib.Module(_lib.shared_codegen([p.text()]), key="cpu_shared_validate")
    ctx = _lib.ExecCtx()
    with pytest.raises(_lib.CxError) as e:
        ctx.shared_execute(m, [], [])
    assert e.value.code == -4  # table rows unset
    plain = _lib.Module(_lib.codegen(p.text()), key="cpu_plain_validate")
    with pytest.raises(_lib.CxError) as e:
        ctx.shared_execute(plain, [], [])
    assert e.value.code == -1


def test_server_config_defaults_and_create_without_a_device():
    cfg = _lib.server_config()
    assert cfg.budget_bytes == 40 << 30 and cfg.max_batch == 64 and cfg.slots == 1 and cfg.plain_only == 0
    assert cfg.min_shared_batch == 5
    assert cfg.shared_tuning.block_threads == 1024
    bad = _lib.server_config(slots=0)
    with pytest.raises(_lib.CxError) as e:
        _lib.Server(_lib.ExecCtx(), bad)
    assert e.value.code in (-1, -7)


def test_parametric_plain_codegen_takes_literals_at_launch():
    rng = random.Random(21)
    t = _lib.default_tuning()
    t.parametric = 1
    a, b = queries.template(2, rng), queries.template(2, rng)
    sa, sb = _lib.codegen(a.text(), t), _lib.codegen(b.text(), t)
    assert sa == sb, "plans of one shape generate one parametric source"
    assert "params 4" in sa and "a.lits" in sa
    m = _lib.Module(sa, key="cpu_param_probe")
    ctx = _lib.ExecCtx()
    with pytest.raises(_lib.CxError) as e:
        ctx.execute(m, 0, [1, 2])  # wrong literal count fails before touching a GPU
    assert e.value.code == -1


def test_bounded_wait_limit_and_stall_hook_reach_the_generated_kernels():
    """Waits are bounded by time (500 ms unless the tuning says otherwise);
    the stall hook is emitted only when asked for, in plain and shared scans."""
    t = _lib.default_tuning()
    assert t.wait_limit_us == 500_000 and t.debug_stall == 0
    plan = queries.ssb_q31()
    t.block_threads, t.stages = 256, 3
    src = _lib.codegen(plan.text(), t)
    assert "debug_stall" not in src and "500000u" in src
    t.wait_limit_us, t.debug_stall = 20_000, 1
    src = _lib.codegen(plan.text(), t)
    assert "cx::debug_stall((unsigned long long*)cx_smem, a.err, 20000u); return;" in src
    _lib.Module(src, key="stall_plain")
    rng = random.Random(5)
    shapes = [queries.template(k, rng).text() for k in range(4)]
    t2 = _lib.default_tuning()
    t2.block_threads, t2.items_per_thread, t2.stages, t2.ctas_per_sm = 1024, 1, 3, 1
    assert "debug_stall" not in _lib.shared_codegen(shapes, t2)
    t2.wait_limit_us, t2.debug_stall = 20_000, 1
    src = _lib.shared_codegen(shapes, t2)
    assert "cx::debug_stall(" in src and "cx::drain_limit_us(" in src
    _lib.Module(src, key="stall_shared")


@pytest.mark.parametrize("name", ["ssb_q31", "ssb_q31_nullable", "T1", "T2", "T3", "kat_q2"])
@pytest.mark.parametrize("ipt", [1, 2, 4, 8])
def test_compacted_scans_compile(name, ipt):
    """Warp compaction: qualifying rows queue per warp; the payload fetches and
    the group update run on 32 queued rows at a time."""
    plan = all_plans()[name]
    t = _lib.default_tuning()
    t.items_per_thread, t.compact = ipt, 1
    if ipt == 8:
        t.block_threads = 512
    src = _lib.codegen(plan.text(), t)
    assert "q_base" in src and "while (q_n >= 32 || (!live_ && q_n > 0))" in src
    _lib.Module(src, key=f"compact_{name}_{ipt}")
    # Two queued batches per drain.
    t.compact = 2
    src2 = _lib.codegen(plan.text(), t)
    assert "while (q_n >= 64 || (!live_ && q_n > 0))" in src2
    _lib.Module(src2, key=f"compact2_{name}_{ipt}")
    t.compact = 1
    # Scalar plans and staged scans keep the direct path.
    t.stages, t.block_threads = 2, 256
    assert "q_base" not in _lib.codegen(plan.text(), t)
    assert "q_base" not in _lib.codegen(all_plans()["ssb_q11"].text(), _lib.default_tuning())


def test_payload_tables_follow_the_catalog_range_and_budget():
    """Joins whose payload has a small catalog range (the plan's prange) keep
    one byte per hash slot in shared memory; a zero budget or an unknown range
    falls back to membership bitmaps and payload loads from the hash table."""
    plan = queries.ssb_q31()
    text = plan.text()
    assert "(prange 1992 7)" in text and "(prange 0 25)" in text
    assert "BlockProbeExactTable" not in _lib.codegen(text)  # opt-in
    on = _lib.default_tuning()
    on.table_budget = 96 * 1024
    src = _lib.codegen(text, on)
    assert src.count("BlockProbeExactTable") == 2      # date (61,131 slots) and supplier (20,000) fit 96 KiB
    assert "BlockProbeExactBitmap" in src             # customer (300,000 slots) keeps its bitmap
    _lib.Module(src, key="ptable_q31")
    t = _lib.default_tuning()
    t.table_budget = 0
    assert "BlockProbeExactTable" not in _lib.codegen(text, t)
    no_range = text.replace("(prange 1992 7)", "").replace("(prange 0 25)", "")
    assert "BlockProbeExactTable" not in _lib.codegen(no_range, on)
    t = _lib.default_tuning()
    t.compact, t.table_budget = 1, 96 * 1024
    src = _lib.codegen(text, t)
    assert "BlockFetchPayloadTable" in src and "q_base" in src
    _lib.Module(src, key="ptable_q31_compact")


def test_cube_scan_region_compiles_with_its_layout_as_constants():
    """The runtime recompiles a shared program's cube region with the batch's
    layout as constants: the region reads its layout only through CXS_*
    macros (defaults: the kernel arguments), and the prelude plus `#define`s
    of every such macro plus the region compile on their own."""
    import re
    from practice_b200.engine import SHARED_DEFAULT, make_tuning
    rng = random.Random(21)
    src = _lib.shared_codegen([queries.template(t, rng).text() for t in range(4)], make_tuning(**SHARED_DEFAULT))
    p0, p1 = src.index("@*/") + 3, src.index("//@cx-prelude-end")
    r0, r1 = src.index("//@cx-cube-begin"), src.index("//@cx-cube-end")
    region = src[r0:r1]
    kernel = region[region.index("#endif"):]
    assert "a.cube_stride[" not in kernel and "a.cube_dsm[" not in kernel  # every layout read is a hook
    defaults = re.findall(r"#define (CXS_\w+) \(a\.(\w+)(?:\[(\d+)\])?\)", region)
    assert defaults
    values = {"cube_dsm": -1, "cube_dgl": 1, "cube_desz": 2, "cube_cells": 1000}
    defs = "#define CXS_SPEC 1\n" + "".join(
        f"#define {name} ({values.get(field, 3)}{'LL' if field == 'cube_cells' else ''})\n" for name, field, _ in defaults)
    spec = "/*@cx-launch\nv 1\n@*/\n" + src[p0:p1] + "\n" + defs + region
    _lib.Module(spec, key="cube_layout_constants")


@pytest.mark.parametrize("bt,ipt,compact", [(1024, 4, 1), (1024, 4, 2), (512, 2, 1), (1024, 8, 2), (256, 1, 1)])
def test_compaction_queue_slots_stay_inside_the_warp_queue(bt, ipt, compact):
    """Every lane computes its queue slot (q_n + its rank among the
    qualifying lanes) and only qualifying lanes store, by predicated stores:
    the slot of every lane must still lie inside its column's queue.  The
    queue layout and the drain size are read from the generated scan; the
    warp's queue is then driven with worst-case ballots (all lanes
    qualifying) and random ones."""
    import random as _random
    import re as _re

    t = _lib.default_tuning()
    t.block_threads, t.items_per_thread, t.compact = bt, ipt, compact
    src = None
    for name in ("ssb_q31_nullable", "T1"):  # the first that fits this launch shape's shared memory
        try:
            src = _lib.codegen(all_plans()[name].text(), t)
            break
        except _lib.CxError:
            continue
    assert src is not None
    offs = sorted(int(x) for x in _re.findall(r"st_shared_if\(f_, &q_base\[(\d+) \+ p_\]", src))
    per_warp = int(_re.search(r"\(long long\)warp \* (\d+)LL; \(void\)q_base;", src).group(1))
    drain = int(_re.search(r"while \(q_n >= (\d+) \|\|", src).group(1))
    assert offs and offs[0] == 0
    cap = offs[1] - offs[0] if len(offs) > 1 else per_warp
    assert all(b - a == cap for a, b in zip(offs, offs[1:])) and offs[-1] + cap == per_warp
    rng = _random.Random(bt * 131 + ipt * 7 + compact)
    for trial in range(200):
        q_n = 0
        for _tile in range(50):
            for _item in range(ipt):
                ballot = 32 if trial % 2 == 0 else rng.choice((0, 1, 5, 31, 32))
                assert q_n + 31 < cap  # the highest slot any lane computes
                q_n += ballot
            while q_n >= drain:
                q_n -= drain
