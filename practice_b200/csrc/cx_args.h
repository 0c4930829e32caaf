// cx_args.h -- the single by-value argument block every generated kernel takes.
//
// The reference binds column pointers by name inside its generated host function
// (`ctx->getBuffer<int>("d_<col>")`, src/core/visitor.cpp:4808-4818).  NVRTC
// compiles device code only, so the generic executor resolves the same names on
// the host and passes them in slots; the launch plan embedded in the generated
// source records which name sits in which slot.  Shared by the host runtime
// (g++) and the NVRTC-compiled kernels, so it holds plain C types only.
#pragma once

#define CX_MAX_COLS 40
#define CX_MAX_HTS 8
#define CX_MAX_TABLES 8
#define CX_MAX_SHAPES 16
#define CX_MAX_FCOLS 8
#define CX_MAX_LITS 64
#define CX_MAX_CATTRS 32
#define CX_MAX_SATTRS 8

// One query of a shared-scan batch: its own result buffers, its plan shape and
// the offset of its literal parameters.
struct CxSQ {
  unsigned long long* result;
  unsigned long long* validity;
  unsigned int* touched;    // per-group "row seen" bits (grouped shapes)
  int shape;
  int param_off;
  int smem_acc;             // u64 offset of its group table in shared memory, -1 = global atomics
  int smem_bits;            // u32 offset of its touched / seen bits in shared memory
  int keep;                 // 1 = add to the result left by earlier row ranges (not zeroed)
};

struct CxArgs {
  const int* col[CX_MAX_COLS];                 // device column bases, by slot
  const unsigned long long* nul[CX_MAX_COLS];  // validity words (1 = valid), by slot
  int* ht[CX_MAX_HTS];                         // perfect hash tables (zeroed before builds)
  unsigned int* htv[CX_MAX_HTS];               // payload validity bits of PHT_2V tables
  unsigned int* bm[CX_MAX_HTS];                // slot-occupancy bits of each hash table
  unsigned long long* result;                  // groups x storage tuple, u64
  unsigned long long* result_validity;         // result validity bits
  unsigned int* touched;                       // per-group "row seen" bits (global group path)
  unsigned long long* finalize_tmp;            // visible tuple staging for AVG finalisation
  unsigned int* err;                           // first error code raised by any kernel
  long long rows[CX_MAX_TABLES];               // row count per plan table slot
  // Shared-scan batches (unused by single-query kernels).
  const struct CxSQ* sq;                       // queries, grouped by shape
  const int* sparams;                          // literal parameters of all queries
  int sq_first[CX_MAX_SHAPES];                 // first query of each shape
  int sq_num[CX_MAX_SHAPES];                   // number of queries of each shape
  int sq_total;
  int nparams;
  int smem_tab_words;                          // u64 words of per-query shared-memory group tables
  int smem_bit_words;                          // u32 words of their touched / seen bits
  int* dat[CX_MAX_HTS];                        // extra payload attributes at each dimension's slots
  int fbase[CX_MAX_FCOLS];                     // first value of each fact filter table window
  int fwin[CX_MAX_FCOLS];                      // values in the window (0: evaluate every row per query)
  int lits[CX_MAX_LITS];                       // literal parameters of a parametric plain kernel
  int* mpay[CX_MAX_HTS];                       // multi-value hash tables: build row ids grouped by slot
  // Aggregate cubes of a shared-scan batch: per attribute the registered range
  // minimum and the number of values; per shape the cell stride of each of its
  // attributes, its cube in global memory (sums per SUM aggregate, then row
  // counts) and the u64 offset of its per-CTA copy in shared memory (-1: none).
  int cube_lo[CX_MAX_CATTRS];
  int cube_radix[CX_MAX_CATTRS];
  int cube_stride[CX_MAX_SHAPES * CX_MAX_SATTRS];
  unsigned long long* cube_g[CX_MAX_SHAPES];
  long long cube_cells[CX_MAX_SHAPES];
  int cube_smem[CX_MAX_SHAPES];
  int cube_smem_words;                         // u64 words of all shared-memory cubes
  int cube_chunks;                             // answer blocks per query
  // An attribute determined by another attribute of the shape (a dimension's
  // functional dependency, e.g. region by nation) takes no part in the cell
  // index: per shape attribute the position of its source attribute in the
  // shape (-1: none), per attribute the table from the source's value offset
  // to its own.
  int cube_fdsrc[CX_MAX_SHAPES * CX_MAX_SATTRS];
  const int* cube_fdtab[CX_MAX_CATTRS];
  // Dimensions whose entries fit in shared memory as compact words (bit 0:
  // a row has this key, then one bit per plan shape, then the attribute
  // offsets), one word per key of the dimension's key range, indexed by
  // key - range minimum (distinct keys, distinct words: no key check): per
  // dimension the byte offset of its copy in shared memory (-1: int4 entries
  // gathered from global memory), the bytes of one word (1, 2 or 4), the key
  // range's minimum and size, the array the index kernel writes, and per
  // attribute field its bit shift and mask.
  int cube_dsm[CX_MAX_HTS];
  int cube_desz[CX_MAX_HTS];
  int cube_dbase[CX_MAX_HTS];
  int cube_dlen[CX_MAX_HTS];
  unsigned char* cube_dcomp[CX_MAX_HTS];
  int cube_fsh[CX_MAX_HTS * 4];
  int cube_fmk[CX_MAX_HTS * 4];
  int cube_dsm_bytes;                          // shared-memory bytes of all compact dimension copies
  int cube_dgl[CX_MAX_HTS];                    // 1: compact words gathered from global memory instead
};
