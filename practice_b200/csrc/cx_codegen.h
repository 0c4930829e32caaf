// cx_codegen.h -- CUDA C++ generation for star-join plans.
#pragma once

#include <string>
#include <vector>

#include "cx_plan.h"

namespace cx {

// Launch shape of the generated fact-scan kernel.  The autotuner searches this
// space per query shape; defaults are the measured best general setting.
struct Tuning {
  int block_threads = 1024;    // BLOCK_THREADS (multiple of 32, <= 1024)
  int items_per_thread = 4;    // ITEMS_PER_THREAD
  int stages = 0;              // TMA staging ring depth (0 disables staging)
  int ctas_per_sm = 16;        // persistent grid = SMs x this (occupancy-capped)
  int group_placement = 0;     // 0 auto, 1 shared-memory tables, 2 global atomics, 3 registers,
                               // 4 per-thread shared-memory tables (<= 16 words per thread)
  int smem_group_budget = 96 * 1024;  // bytes of shared memory a group table may use
  int bitmap_budget = 48 * 1024;      // bytes of shared memory for join membership bitmaps
  int group_merge = 0;         // 0 auto, 1 warp match-merge (one expanding join: warp-uniform
                               // expansion), 2 direct per-lane atomics, 3 shared scans: direct
                               // per-row atomics above 32 groups only
  int producer_warps = 0;      // shared scans: warps that build query masks (0 = 3/8 of the block)
  int parametric = 0;          // plain kernels: literals read from CxArgs.lits at run time
  int prefetch = 1;            // unstaged plain scans: 0 columns loaded where first used,
                               // 1 vector loads of every column at the tile start,
                               // 2 as 1 and the next tile's loads issued one tile ahead,
                               // 3 as 1 and an L2 bulk prefetch of the warp's next tile
  int wait_limit_us = 500000;  // a bounded mbarrier wait gives up after this many microseconds
  int debug_stall = 0;         // test hook: 1 = every CTA first waits on a barrier nothing completes
  int compact = 0;             // plain grouped scans: 1 = queue qualifying rows per warp after the
                               // membership tests and run the rest on 32 queued rows at a time
  int table_budget = 0;        // bytes of shared memory for payload tables (one byte per slot); opt-in:
                               // measured no faster than bitmaps once rows are warp-compacted
  int cube = 4;                // shared scans: 0 = per-query row masks only; 1, 2 or 4 = also the
                               // aggregate-cube path (rows per lane of its scan), which the runtime
                               // takes when the batch's attribute ranges allow
};

// Returns the CUDA source for `plan` with its launch plan embedded as a
// leading `/*@cx-launch ... @*/` block.  Throws PlanError on unsupported shapes.
std::string generate_cuda(const Plan& plan, const Tuning& tuning);

// The integer literals of a plan in the canonical order that numbers the
// parameters of its shape (steps, then GROUP BY, then aggregates; pre-order).
void collect_literals(const Plan& plan, std::vector<const Expr*>& out);

// Shared-scan kernel for a set of plan shapes (one representative plan per
// shape; literals become per-query parameters).  Throws PlanError when a shape
// cannot share a scan (nullable columns, AVG/MIN/MAX, > 3 attributes of one
// dimension, conflicting joins, literals outside int32).
std::string generate_shared_cuda(const std::vector<const Plan*>& shapes, const Tuning& tuning);

// Whether one plan shape can join a shared scan (the checks of
// generate_shared_cuda without generating code); `why` gets the reason if not.
bool shared_shape_ok(const Plan& plan, std::string* why);

}  // namespace cx
