/* crystal_oracle.c -- CPU restatement of crystal-sycl's fused star-join query
 * pipeline, used ONLY as the test oracle (and as the bench's CPU baseline leg).
 * It is test infrastructure: the product path (libcrystal_b200.so) never links,
 * loads or calls it.
 *
 * Input: the same star-join plan text the code generator reads (see
 * practice_b200/csrc/cx_plan.h), plus host column arrays.  Output: the raw
 * aggregate buffer (groups x storage tuple of u64) and its validity bitmap, in
 * exactly the state the reference's generated execute_query leaves them before
 * result materialisation.
 *
 * Semantics restated from the reference (paths inside the reference project):
 *   build     include/crystal/join.h:124-253   CAS(ht[h], 0, key); PHT_2 also
 *             stores ht[2h+1] = payload after the CAS, whatever its outcome.
 *   probe     include/crystal/join.h:7-120     ht[h] == key (PHT_1),
 *             ht[2h] == key -> payload (PHT_2); h = (key - key_min) % len.
 *   filters   src/core/visitor.cpp:921-991, 1218-1489  three-valued logic:
 *             a row passes when the predicate is known (valid) and true; AND is
 *             known when either side is known false or both are known; OR
 *             when either side is known true or both are known.
 *   predicate arithmetic and comparisons promote int32 to int64
 *             (include/core/inline_math.h:15-94).
 *   aggregate inputs   src/core/visitor.cpp:1947-2010 (translateMathExprPush):
 *             only the leftmost leaf is widened to unsigned 64-bit; right
 *             operands keep their C types (int32 arithmetic wraps).
 *   aggregates  scalar :3017-3124, grouped :3125-3195, MIN slots start at ~0
 *             (:2474-2503), AVG finalisation (:2505-2586).
 *   group hash  :2056-2127  Horner over (value - min) terms; a nullable key
 *             maps NULL to 0 and shifts values by +1; result % product.
 *   validity bits  set exactly where the reference calls atomic_set_valid_bit.
 *
 * Three documented choices where the reference is undefined or racy:
 *   - a slot outside [0, len) misses / is skipped (reference: out of bounds);
 *   - integer division by zero yields 0 (reference: undefined behaviour);
 *   - the key slot of a NULL GROUP BY key holds 0 (reference: the raw value
 *     of whichever row wrote last, behind a cleared validity bit).
 *   Group-key slots hold the key values of the group; rows whose key lies
 *   outside its catalog domain raise an error count (reference: silent fold).
 *   Nullable join payloads keep their validity through the hash table (the
 *   reference drops it, src/core/visitor.cpp:4577-4578).
 */
#include <ctype.h>
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXK 64

/* ------------------------------------------------------------- s-expr --- */
typedef struct Node {
  int atom;
  char* text;
  struct Node** items;
  int n;
} Node;

typedef struct {
  const char* s;
  size_t pos, len;
  char err[256];
} Reader;

static void skip(Reader* r) {
  while (r->pos < r->len) {
    char c = r->s[r->pos];
    if (isspace((unsigned char)c)) r->pos++;
    else if (c == ';') { while (r->pos < r->len && r->s[r->pos] != '\n') r->pos++; }
    else break;
  }
}

static Node* read_node(Reader* r) {
  skip(r);
  if (r->pos >= r->len) { snprintf(r->err, sizeof r->err, "unexpected end"); return NULL; }
  Node* n = (Node*)calloc(1, sizeof(Node));
  if (r->s[r->pos] == '(') {
    r->pos++;
    int cap = 4;
    n->items = (Node**)malloc(sizeof(Node*) * cap);
    for (;;) {
      skip(r);
      if (r->pos >= r->len) { snprintf(r->err, sizeof r->err, "missing )"); return NULL; }
      if (r->s[r->pos] == ')') { r->pos++; break; }
      Node* k = read_node(r);
      if (!k) return NULL;
      if (n->n == cap) { cap *= 2; n->items = (Node**)realloc(n->items, sizeof(Node*) * cap); }
      n->items[n->n++] = k;
    }
    return n;
  }
  size_t b = r->pos;
  while (r->pos < r->len && !isspace((unsigned char)r->s[r->pos]) && r->s[r->pos] != '(' && r->s[r->pos] != ')') r->pos++;
  n->atom = 1;
  n->text = (char*)malloc(r->pos - b + 1);
  memcpy(n->text, r->s + b, r->pos - b);
  n->text[r->pos - b] = 0;
  return n;
}

static void free_node(Node* n) {
  if (!n) return;
  for (int i = 0; i < n->n; ++i) free_node(n->items[i]);
  free(n->items);
  free(n->text);
  free(n);
}

static const char* head(const Node* n) {
  if (!n || n->atom || n->n == 0 || !n->items[0]->atom) return "";
  return n->items[0]->text;
}

static const Node* field(const Node* n, const char* key) {
  for (int i = 1; i < n->n; ++i)
    if (strcmp(head(n->items[i]), key) == 0) return n->items[i];
  return NULL;
}

/* ------------------------------------------------------------- plan --- */
enum { E_COL, E_INT, E_NULL, E_STAR, E_ADD, E_SUB, E_MUL, E_DIV, E_EQ, E_NE, E_LT, E_LE, E_GT, E_GE,
       E_AND, E_OR, E_NOT, E_ISNULL, E_NOTNULL, E_CASE };

typedef struct Expr {
  int op;
  int col;          /* column index into the oracle's column table */
  long long ival;
  struct Expr* k[3];
} Expr;

/* Column registry. */
typedef struct {
  char name[64];
  const int32_t* data;
  const uint64_t* valid;  /* may be NULL: all valid */
  int nullable;           /* catalog-nullable */
  int table;
  int is_payload;         /* set when a join publishes it */
} Col;

typedef struct {
  int dim_table;
  int pk, payload;      /* column ids, payload -1 for PHT_1 */
  int fks[4], nfk;      /* probe keys; more than one is an OR-join */
  int multi;            /* multi-value hash table (non-unique build key) */
  int gathers[8], ngather; /* MHT: build columns read through the row id */
  long long len, keymin;
  Expr* filter;
  int32_t* ht;          /* 2*len ints */
  unsigned char* hv;    /* payload validity per slot (nullable payloads) */
  int32_t* mkey;        /* MHT directory: key, count and first position per slot */
  int32_t* mcnt;
  long long* moff;
  int32_t* mrows;       /* MHT payload: build row ids grouped by slot */
} JoinS;

typedef struct {
  int kind; /* 0 filter, 1 join */
  Expr* filter;
  JoinS join;
} StepS;

typedef struct {
  Expr* e;
  long long min, card;
  int nullable;
} GroupS;

typedef struct {
  int fn; /* 0 count 1 sum 2 min 3 max 4 avg */
  Expr* arg;
} AggS;

typedef struct {
  char tables[8][64];
  int ntables;
  long long rows[8];
  Col cols[256];
  int ncols;
  StepS steps[32];
  int nsteps;
  GroupS groups[16];
  int ngroups;
  AggS aggs[32];
  int naggs;
  int sparse;
  char err[512];
  /* per-row state for the scan */
  int32_t* payload_val;   /* per column: current row's payload value */
  int* payload_valid;
} Oracle;

static int col_index(Oracle* o, const char* name) {
  for (int i = 0; i < o->ncols; ++i)
    if (strcmp(o->cols[i].name, name) == 0) return i;
  return -1;
}

static Expr* to_expr(Oracle* o, const Node* n) {
  const char* h = head(n);
  Expr* e = (Expr*)calloc(1, sizeof(Expr));
  static const struct { const char* name; int op; int ar; } ops[] = {
      {"add", E_ADD, 2}, {"sub", E_SUB, 2}, {"mul", E_MUL, 2}, {"div", E_DIV, 2}, {"eq", E_EQ, 2},
      {"ne", E_NE, 2},   {"lt", E_LT, 2},   {"le", E_LE, 2},   {"gt", E_GT, 2},   {"ge", E_GE, 2},
      {"and", E_AND, 2}, {"or", E_OR, 2},   {"not", E_NOT, 1}, {"isnull", E_ISNULL, 1},
      {"notnull", E_NOTNULL, 1}, {"case", E_CASE, 3}};
  if (!strcmp(h, "col")) {
    e->op = E_COL;
    e->col = col_index(o, n->items[1]->text);
    if (e->col < 0) { snprintf(o->err, sizeof o->err, "unknown column %s", n->items[1]->text); return NULL; }
    return e;
  }
  if (!strcmp(h, "int")) { e->op = E_INT; e->ival = strtoll(n->items[1]->text, NULL, 10); return e; }
  if (!strcmp(h, "null")) { e->op = E_NULL; return e; }
  if (!strcmp(h, "star")) { e->op = E_STAR; return e; }
  for (size_t i = 0; i < sizeof ops / sizeof ops[0]; ++i) {
    if (!strcmp(h, ops[i].name)) {
      e->op = ops[i].op;
      if (n->n != ops[i].ar + 1) { snprintf(o->err, sizeof o->err, "arity of %s", h); return NULL; }
      for (int k = 0; k < ops[i].ar; ++k) {
        e->k[k] = to_expr(o, n->items[k + 1]);
        if (!e->k[k]) return NULL;
      }
      return e;
    }
  }
  snprintf(o->err, sizeof o->err, "unknown expression %s", h);
  return NULL;
}

static void free_expr(Expr* e) {
  if (!e) return;
  for (int i = 0; i < 3; ++i) free_expr(e->k[i]);
  free(e);
}

/* ---------------------------------------------------------- evaluation --- */
/* Typed values of the C expressions the reference generates. */
enum { T_I32, T_I64, T_U64 };
typedef struct { int t; uint64_t bits; } TV;

static int64_t as_i64(TV v) {
  if (v.t == T_I32) return (int64_t)(int32_t)(uint32_t)v.bits;
  return (int64_t)v.bits;
}
static TV mk(int t, uint64_t bits) {
  TV v;
  v.t = t;
  v.bits = (t == T_I32) ? (uint64_t)(uint32_t)bits : bits;
  return v;
}
static TV convert(TV v, int t) {
  if (v.t == t) return v;
  if (t == T_I32) return mk(T_I32, (uint32_t)v.bits);
  return mk(t, (uint64_t)as_i64(v)); /* widen with sign extension (I32 -> I64/U64, I64 -> U64) */
}
static int promote(int a, int b) {
  if (a == T_U64 || b == T_U64) return T_U64;
  if (a == T_I64 || b == T_I64) return T_I64;
  return T_I32;
}
static TV arith(int op, TV l, TV r) {
  const int t = promote(l.t, r.t);
  l = convert(l, t);
  r = convert(r, t);
  if (t == T_I32) {
    uint32_t a = (uint32_t)l.bits, b = (uint32_t)r.bits;
    switch (op) {
      case E_ADD: return mk(t, a + b);
      case E_SUB: return mk(t, a - b);
      case E_MUL: return mk(t, a * b);
      default: {
        int32_t x = (int32_t)a, y = (int32_t)b;
        if (y == 0) return mk(t, 0);
        if (x == INT32_MIN && y == -1) return mk(t, (uint32_t)x);
        return mk(t, (uint32_t)(x / y));
      }
    }
  }
  if (t == T_I64) {
    uint64_t a = l.bits, b = r.bits;
    switch (op) {
      case E_ADD: return mk(t, a + b);
      case E_SUB: return mk(t, a - b);
      case E_MUL: return mk(t, a * b);
      default: {
        int64_t x = (int64_t)a, y = (int64_t)b;
        if (y == 0) return mk(t, 0);
        if (x == INT64_MIN && y == -1) return mk(t, (uint64_t)x);
        return mk(t, (uint64_t)(x / y));
      }
    }
  }
  switch (op) {
    case E_ADD: return mk(t, l.bits + r.bits);
    case E_SUB: return mk(t, l.bits - r.bits);
    case E_MUL: return mk(t, l.bits * r.bits);
    default: return mk(t, r.bits == 0 ? 0 : l.bits / r.bits);
  }
}
static int compare(int op, TV l, TV r) {
  const int t = promote(l.t == T_I32 ? T_I64 : l.t, r.t == T_I32 ? T_I64 : r.t);
  int c;
  if (t == T_U64) {
    uint64_t a = convert(l, T_U64).bits, b = convert(r, T_U64).bits;
    c = a < b ? -1 : a > b ? 1 : 0;
  } else {
    int64_t a = as_i64(l), b = as_i64(r);
    c = a < b ? -1 : a > b ? 1 : 0;
  }
  switch (op) {
    case E_EQ: return c == 0;
    case E_NE: return c != 0;
    case E_LT: return c < 0;
    case E_LE: return c <= 0;
    case E_GT: return c > 0;
    default: return c >= 0;
  }
}

typedef struct {
  Oracle* o;
  long long row;      /* fact row */
} RowCtx;

static int col_value(RowCtx* rc, int c, int* valid) {
  Col* col = &rc->o->cols[c];
  if (col->is_payload) {
    *valid = rc->o->payload_valid[c];
    return rc->o->payload_val[c];
  }
  const long long r = rc->row;
  *valid = col->valid ? (int)((col->valid[r >> 6] >> (r & 63)) & 1ULL) : 1;
  if (!col->nullable) *valid = 1;
  return col->data[r];
}

static int valid_of(RowCtx* rc, const Expr* e);
static TV value_of(RowCtx* rc, const Expr* e);

/* expressionValidExpr (src/core/visitor.cpp:921-991). */
static int valid_of(RowCtx* rc, const Expr* e) {
  int v;
  switch (e->op) {
    case E_NULL: return 0;
    case E_STAR: case E_INT: case E_ISNULL: case E_NOTNULL: return 1;
    case E_COL: col_value(rc, e->col, &v); return v;
    case E_NOT: return valid_of(rc, e->k[0]);
    case E_AND: {
      int lv = valid_of(rc, e->k[0]), rv = valid_of(rc, e->k[1]);
      int l = value_of(rc, e->k[0]).bits != 0, r = value_of(rc, e->k[1]).bits != 0;
      return (lv && !l) || (rv && !r) || (lv && rv);
    }
    case E_OR: {
      int lv = valid_of(rc, e->k[0]), rv = valid_of(rc, e->k[1]);
      int l = value_of(rc, e->k[0]).bits != 0, r = value_of(rc, e->k[1]).bits != 0;
      return (lv && l) || (rv && r) || (lv && rv);
    }
    case E_CASE: {
      int sel = valid_of(rc, e->k[0]) && value_of(rc, e->k[0]).bits != 0;
      return sel ? valid_of(rc, e->k[1]) : valid_of(rc, e->k[2]);
    }
    default: return valid_of(rc, e->k[0]) && valid_of(rc, e->k[1]);
  }
}

/* expressionValueNoEmit (:890-920); arithmetic and compares via db::safe_*. */
static TV value_of(RowCtx* rc, const Expr* e) {
  int v;
  switch (e->op) {
    case E_COL: return mk(T_I32, (uint32_t)col_value(rc, e->col, &v));
    case E_INT: return (e->ival >= -2147483647LL && e->ival <= 2147483647LL) ? mk(T_I32, (uint32_t)(int32_t)e->ival)
                                                                               : mk(T_I64, (uint64_t)e->ival);
    case E_NULL: return mk(T_I32, 0);
    case E_STAR: return mk(T_I32, 1);
    case E_ISNULL: return mk(T_I32, !valid_of(rc, e->k[0]));
    case E_NOTNULL: return mk(T_I32, valid_of(rc, e->k[0]));
    case E_NOT: return mk(T_I32, value_of(rc, e->k[0]).bits == 0);
    case E_AND: return mk(T_I32, value_of(rc, e->k[0]).bits != 0 && value_of(rc, e->k[1]).bits != 0);
    case E_OR: return mk(T_I32, value_of(rc, e->k[0]).bits != 0 || value_of(rc, e->k[1]).bits != 0);
    case E_CASE: {
      TV a = value_of(rc, e->k[1]), b = value_of(rc, e->k[2]);
      const int t = promote(a.t, b.t);
      int sel = valid_of(rc, e->k[0]) && value_of(rc, e->k[0]).bits != 0;
      return convert(sel ? a : b, t);
    }
    case E_ADD: case E_SUB: case E_MUL: case E_DIV: {
      TV l = value_of(rc, e->k[0]), r = value_of(rc, e->k[1]);
      if (l.t == T_I32) l = convert(l, T_I64);
      if (r.t == T_I32) r = convert(r, T_I64);
      return arith(e->op, l, r);
    }
    default:
      return mk(T_I32, compare(e->op, value_of(rc, e->k[0]), value_of(rc, e->k[1])));
  }
}

/* translateMathExprPush (:1947-2010): leftmost leaf widened when cast. */
static TV math_push(RowCtx* rc, const Expr* e, int cast) {
  int v;
  switch (e->op) {
    case E_COL: {
      int x = col_value(rc, e->col, &v);
      return cast ? mk(T_U64, (uint64_t)(int64_t)x) : mk(T_I32, (uint32_t)x);
    }
    case E_INT: return (e->ival >= -2147483647LL && e->ival <= 2147483647LL) ? mk(T_I32, (uint32_t)(int32_t)e->ival)
                                                                               : mk(T_I64, (uint64_t)e->ival);
    case E_STAR: return cast ? mk(T_U64, 1) : mk(T_I32, 1);
    case E_NULL: return mk(T_I32, 0);
    case E_ADD: case E_SUB: case E_MUL: case E_DIV:
      return arith(e->op, math_push(rc, e->k[0], cast), math_push(rc, e->k[1], 0));
    default: {
      TV x = value_of(rc, e);
      return cast ? convert(x, T_U64) : x;
    }
  }
}

static int passes(RowCtx* rc, const Expr* e) { return valid_of(rc, e) && value_of(rc, e).bits != 0; }

/* --------------------------------------------------------------- driver --- */
static int parse(Oracle* o, const char* text) {
  Reader rd = {text, 0, strlen(text), {0}};
  Node* root = read_node(&rd);
  if (!root) { snprintf(o->err, sizeof o->err, "parse: %s", rd.err); return -1; }
  if (strcmp(head(root), "query")) { snprintf(o->err, sizeof o->err, "not a (query ...)"); free_node(root); return -1; }
  int rc = 0;
  /* pass 1: tables + columns; fact table goes first */
  for (int pass = 0; pass < 2; ++pass)
    for (int i = 1; i < root->n; ++i) {
      const Node* n = root->items[i];
      if (strcmp(head(n), "table")) continue;
      int fact = 0;
      const Node* cols = NULL;
      for (int k = 2; k < n->n; ++k) {
        if (n->items[k]->atom && !strcmp(n->items[k]->text, "fact")) fact = 1;
        else if (!strcmp(head(n->items[k]), "cols")) cols = n->items[k];
      }
      if (fact != (pass == 0)) continue;
      const int t = o->ntables++;
      snprintf(o->tables[t], sizeof o->tables[t], "%s", n->items[1]->text);
      for (int c = 1; cols && c < cols->n; ++c) {
        Col* cl = &o->cols[o->ncols++];
        memset(cl, 0, sizeof *cl);
        snprintf(cl->name, sizeof cl->name, "%s", cols->items[c]->text);
        cl->table = t;
      }
    }
  for (int i = 1; i < root->n && !rc; ++i) {
    const Node* n = root->items[i];
    const char* h = head(n);
    if (!strcmp(h, "nullable")) {
      for (int k = 1; k < n->n; ++k) {
        int c = col_index(o, n->items[k]->text);
        if (c >= 0) o->cols[c].nullable = 1;
      }
    }
  }
  for (int i = 1; i < root->n && !rc; ++i) {
    const Node* n = root->items[i];
    const char* h = head(n);
    if (!strcmp(h, "filter")) {
      StepS* s = &o->steps[o->nsteps++];
      s->kind = 0;
      s->filter = to_expr(o, n->items[1]);
      if (!s->filter) rc = -1;
    } else if (!strcmp(h, "join")) {
      StepS* s = &o->steps[o->nsteps++];
      s->kind = 1;
      JoinS* j = &s->join;
      j->dim_table = -1;
      for (int t = 0; t < o->ntables; ++t)
        if (!strcmp(o->tables[t], n->items[1]->text)) j->dim_table = t;
      j->pk = col_index(o, field(n, "pk")->items[1]->text);
      const Node* fkn = field(n, "fk");
      int bad = fkn->n < 2 || fkn->n > 5;
      for (int k = 1; k < fkn->n && k <= 4; ++k) {
        j->fks[j->nfk] = col_index(o, fkn->items[k]->text);
        bad |= j->fks[j->nfk++] < 0;
      }
      j->len = strtoll(field(n, "len")->items[1]->text, NULL, 10);
      j->keymin = strtoll(field(n, "keymin")->items[1]->text, NULL, 10);
      const Node* mu = field(n, "multi");
      j->multi = mu ? atoi(mu->items[1]->text) != 0 : 0;
      const Node* f = field(n, "filter");
      j->filter = f ? to_expr(o, f->items[1]) : NULL;
      const Node* p = field(n, "payload");
      j->payload = -1;
      if (p && j->multi) {
        for (int k = 1; k < p->n && k <= 8; ++k) {
          j->gathers[j->ngather] = col_index(o, p->items[k]->text);
          bad |= j->gathers[j->ngather++] < 0;
        }
      } else if (p) {
        j->payload = col_index(o, p->items[1]->text);
        bad |= j->payload < 0;
      }
      if (j->dim_table < 0 || j->pk < 0 || bad || (f && !j->filter)) {
        snprintf(o->err, sizeof o->err, "bad join");
        rc = -1;
      }
    } else if (!strcmp(h, "aggregate")) {
      for (int k = 1; k < n->n && !rc; ++k) {
        const Node* a = n->items[k];
        const char* ah = head(a);
        if (!strcmp(ah, "group")) {
          GroupS* g = &o->groups[o->ngroups++];
          g->e = to_expr(o, a->items[1]);
          g->min = strtoll(field(a, "min")->items[1]->text, NULL, 10);
          g->card = strtoll(field(a, "card")->items[1]->text, NULL, 10);
          const Node* nl = field(a, "nullable");
          g->nullable = nl ? atoi(nl->items[1]->text) : 0;
          if (!g->e) rc = -1;
        } else if (!strcmp(ah, "sparse")) {
          o->sparse = atoi(a->items[1]->text);
        } else {
          AggS* g = &o->aggs[o->naggs++];
          g->fn = !strcmp(ah, "count") ? 0 : !strcmp(ah, "sum") ? 1 : !strcmp(ah, "min") ? 2 : !strcmp(ah, "max") ? 3 : 4;
          g->arg = to_expr(o, a->items[1]);
          if (!g->arg) rc = -1;
        }
      }
    }
  }
  free_node(root);
  return rc;
}

static void set_bit(uint64_t* bm, uint64_t bit) { bm[bit >> 6] |= 1ULL << (bit & 63); }
static int get_bit(const uint64_t* bm, uint64_t bit) { return (int)((bm[bit >> 6] >> (bit & 63)) & 1ULL); }

/* Aggregation state of the scan. */
typedef struct {
  Oracle* o;
  uint64_t* result;
  uint64_t* validity;
  uint64_t G;
  int ts, vts;
  uint64_t acc[32], seen[32], cnt[32];
  unsigned char* touched;
  long long derr;
} ScanState;

/* One qualifying (expanded) row into the aggregate: scalar :3017-3124,
 * grouped :3125-3195. */
static void consume(ScanState* st, RowCtx* rcx) {
  Oracle* o = st->o;
  if (o->ngroups == 0) {
    for (int a = 0; a < o->naggs; ++a) {
      const AggS* ag = &o->aggs[a];
      const int v = ag->arg->op == E_STAR ? 1 : valid_of(rcx, ag->arg);
      if (!v) continue;
      const uint64_t x = ag->fn == 0 ? 1 : convert(math_push(rcx, ag->arg, 1), T_U64).bits;
      switch (ag->fn) {
        case 0: st->acc[a] += 1; break;
        case 1: st->acc[a] += x; st->seen[a]++; break;
        case 4: st->acc[a] += x; st->cnt[a]++; break;
        case 2: if (x < st->acc[a]) st->acc[a] = x; st->seen[a]++; break;
        case 3: if (x > st->acc[a]) st->acc[a] = x; st->seen[a]++; break;
      }
    }
    return;
  }
  /* Grouped: perfect hash. */
  long long hsh = 0;
  int dom_ok = 1;
  for (int g = 0; g < o->ngroups; ++g) {
    const GroupS* gs = &o->groups[g];
    const long long card = gs->card + (gs->nullable ? 1 : 0);
    long long term;
    const int64_t v = as_i64(value_of(rcx, gs->e));
    if (gs->nullable) term = valid_of(rcx, gs->e) ? v - gs->min + 1 : 0;
    else term = v - gs->min;
    if (term < 0 || term >= card) dom_ok = 0;
    hsh = g == 0 ? term : hsh * card + term;
  }
  hsh = hsh % (long long)st->G;
  if (!dom_ok) st->derr++;
  if (hsh < 0 || (uint64_t)hsh >= st->G) return;
  const uint64_t base = (uint64_t)hsh * st->ts;
  uint64_t* result = st->result;
  st->touched[hsh] = 1;
  int avg_i = 0;
  for (int a = 0; a < o->naggs; ++a) {
    const AggS* ag = &o->aggs[a];
    const int slot = o->ngroups + a;
    const int v = ag->arg->op == E_STAR ? 1 : valid_of(rcx, ag->arg);
    if (ag->fn == 0) {
      if (v) result[base + slot] += 1;
      if (!o->sparse) set_bit(st->validity, base + slot);
      continue;
    }
    if (ag->fn == 4) {
      if (v) {
        result[base + slot] += convert(math_push(rcx, ag->arg, 1), T_U64).bits;
        result[base + st->vts + avg_i] += 1;
      }
      avg_i++;
      continue;
    }
    if (!v) continue;
    const uint64_t x = convert(math_push(rcx, ag->arg, 1), T_U64).bits;
    if (ag->fn == 1) result[base + slot] += x;
    else if (ag->fn == 2) { if (x < result[base + slot]) result[base + slot] = x; }
    else { if (x > result[base + slot]) result[base + slot] = x; }
    if (!o->sparse) set_bit(st->validity, base + slot);
  }
}

/* PHT probe of one key; publishes the payload on a hit (join.h:43-120). */
static int probe_pht(Oracle* o, JoinS* j, int fk) {
  const long long h = ((long long)fk - j->keymin) % j->len;
  if (h < 0 || h >= j->len) return 0;
  if (j->payload < 0) return j->ht[h] == fk;
  if (j->ht[2 * h] != fk) return 0;
  o->payload_val[j->payload] = j->ht[2 * h + 1];
  o->payload_valid[j->payload] = o->cols[j->payload].nullable ? j->hv[h] : 1;
  return 1;
}

/* Runs pipeline steps s.. for the current fact row.  An expanding join (an
 * OR over several fact keys, visitor.cpp:4587-4640, or an MHT probe,
 * :4672-4730) runs the rest of the pipeline once per distinct non-NULL key
 * (a key equal to an earlier valid key of the row is skipped) and, for an
 * MHT, once per matching build row. */
static void walk(ScanState* st, RowCtx* rcx, int s) {
  Oracle* o = st->o;
  for (; s < o->nsteps; ++s) {
    StepS* sp = &o->steps[s];
    if (sp->kind == 0) {
      if (!passes(rcx, sp->filter)) return;
      continue;
    }
    JoinS* j = &sp->join;
    if (j->nfk == 1 && !j->multi) {
      int fv;
      const int fk = col_value(rcx, j->fks[0], &fv);
      if (!fv || !probe_pht(o, j, fk)) return;
      continue;
    }
    for (int f = 0; f < j->nfk; ++f) {
      int fv;
      const int fk = col_value(rcx, j->fks[f], &fv);
      if (!fv) continue;
      int dup = 0;
      for (int q = 0; q < f; ++q) {
        int pv;
        const int pk = col_value(rcx, j->fks[q], &pv);
        if (pv && pk == fk) dup = 1;
      }
      if (dup) continue;
      if (!j->multi) {
        if (probe_pht(o, j, fk)) walk(st, rcx, s + 1);
        continue;
      }
      const long long h = ((long long)fk - j->keymin) % j->len;
      if (h < 0 || h >= j->len || j->mcnt[h] == 0 || j->mkey[h] != fk) continue;
      for (long long k = 0; k < j->mcnt[h]; ++k) {
        const long long rid = j->mrows[j->moff[h] + k];
        for (int g = 0; g < j->ngather; ++g) {
          const Col* c = &o->cols[j->gathers[g]];
          o->payload_val[j->gathers[g]] = c->data[rid];
          o->payload_valid[j->gathers[g]] =
              (c->nullable && c->valid) ? (int)((c->valid[rid >> 6] >> (rid & 63)) & 1ULL) : 1;
        }
        walk(st, rcx, s + 1);
      }
    }
    return;
  }
  consume(st, rcx);
}

/* Evaluates a plan over host columns.  Returns 0, or -1 with `err` filled.
 * `domain_errors` receives the number of rows whose GROUP BY key fell outside
 * its catalog domain. */
int oracle_run(const char* plan, int ncol, const char* const* names, const int32_t* const* data,
               const uint64_t* const* valid, int ntab, const char* const* tnames, const long long* trows,
               uint64_t* result, uint64_t result_words, uint64_t* validity, uint64_t validity_words,
               long long* domain_errors, char* err, int errlen) {
  Oracle* o = (Oracle*)calloc(1, sizeof(Oracle));
  int rc = parse(o, plan);
  if (rc) goto done;
  for (int i = 0; i < o->ncols; ++i) {
    for (int k = 0; k < ncol; ++k)
      if (!strcmp(names[k], o->cols[i].name)) { o->cols[i].data = data[k]; o->cols[i].valid = valid[k]; }
  }
  for (int t = 0; t < o->ntables; ++t) {
    o->rows[t] = -1;
    for (int k = 0; k < ntab; ++k)
      if (!strcmp(tnames[k], o->tables[t])) o->rows[t] = trows[k];
    if (o->rows[t] < 0) { snprintf(o->err, sizeof o->err, "rows of %s missing", o->tables[t]); rc = -1; goto done; }
  }
  o->payload_val = (int32_t*)calloc(o->ncols, sizeof(int32_t));
  o->payload_valid = (int*)calloc(o->ncols, sizeof(int));

  /* Layout. */
  uint64_t G = 1;
  for (int g = 0; g < o->ngroups; ++g) G *= (uint64_t)(o->groups[g].card + (o->groups[g].nullable ? 1 : 0));
  int navg = 0;
  for (int a = 0; a < o->naggs; ++a) navg += o->aggs[a].fn == 4;
  int ts = o->ngroups + o->naggs + navg;
  if (ts == 0) ts = 1;
  const int vts = o->ngroups + o->naggs;
  if (result_words < G * (uint64_t)ts || validity_words < (G * ts + 63) / 64) {
    snprintf(o->err, sizeof o->err, "result buffers too small");
    rc = -1;
    goto done;
  }
  memset(result, 0, result_words * 8);
  memset(validity, 0, validity_words * 8);
  for (uint64_t g = 0; g < G; ++g)
    for (int a = 0; a < o->naggs; ++a)
      if (o->aggs[a].fn == 2) result[g * ts + o->ngroups + a] = ~0ULL; /* init_aggregate_slots */

  /* Builds, in plan order (the reference emits them before the scan). */
  for (int s = 0; s < o->nsteps; ++s) {
    if (o->steps[s].kind != 1) continue;
    JoinS* j = &o->steps[s].join;
    for (int i = 0; i < o->ncols; ++i)
      if (!o->cols[i].data && o->cols[i].table == j->dim_table) { snprintf(o->err, sizeof o->err, "column %s has no data", o->cols[i].name); rc = -1; goto done; }
    const long long n = o->rows[j->dim_table];
    RowCtx rcx = {o, 0};
    if (j->multi) {
      /* MHT build (visitor.cpp:4295-4464): count per slot, exclusive prefix
       * sum, then row ids grouped by slot (ascending here; the device order
       * within a slot is unspecified and aggregation does not depend on it).
       * Two distinct keys in one slot are an error (the reference merges them
       * into one directory entry under whichever key was written last). */
      j->mkey = (int32_t*)calloc((size_t)j->len, sizeof(int32_t));
      j->mcnt = (int32_t*)calloc((size_t)j->len, sizeof(int32_t));
      j->moff = (long long*)calloc((size_t)j->len + 1, sizeof(long long));
      for (long long r = 0; r < n; ++r) {
        rcx.row = r;
        if (j->filter && !passes(&rcx, j->filter)) continue;
        int kv;
        const int key = col_value(&rcx, j->pk, &kv);
        if (!kv) continue;
        const long long h = ((long long)key - j->keymin) % j->len;
        if (h < 0 || h >= j->len) continue;
        if (j->mcnt[h] && j->mkey[h] != key) { snprintf(o->err, sizeof o->err, "MHT slot collision in %s", o->tables[j->dim_table]); rc = -1; goto done; }
        j->mkey[h] = key;
        j->mcnt[h]++;
      }
      for (long long h = 0; h < j->len; ++h) j->moff[h + 1] = j->moff[h] + j->mcnt[h];
      j->mrows = (int32_t*)calloc((size_t)j->moff[j->len] + 1, sizeof(int32_t));
      long long* pos = (long long*)calloc((size_t)j->len, sizeof(long long));
      for (long long r = 0; r < n; ++r) {
        rcx.row = r;
        if (j->filter && !passes(&rcx, j->filter)) continue;
        int kv;
        const int key = col_value(&rcx, j->pk, &kv);
        if (!kv) continue;
        const long long h = ((long long)key - j->keymin) % j->len;
        if (h < 0 || h >= j->len) continue;
        j->mrows[j->moff[h] + pos[h]++] = (int32_t)r;
      }
      free(pos);
      for (int g = 0; g < j->ngather; ++g) o->cols[j->gathers[g]].is_payload = 1;
      continue;
    }
    j->ht = (int32_t*)calloc((size_t)(2 * j->len), sizeof(int32_t));
    j->hv = (unsigned char*)calloc((size_t)j->len, 1);
    for (long long r = 0; r < n; ++r) {
      rcx.row = r;
      if (j->filter && !passes(&rcx, j->filter)) continue;
      int kv;
      const int key = col_value(&rcx, j->pk, &kv);
      if (!kv) continue;
      const long long h = ((long long)key - j->keymin) % j->len;
      if (h < 0 || h >= j->len) continue;
      if (j->payload < 0) {
        if (j->ht[h] == 0) j->ht[h] = key;
      } else {
        if (j->ht[2 * h] == 0) j->ht[2 * h] = key;
        int pv;
        j->ht[2 * h + 1] = col_value(&rcx, j->payload, &pv);
        j->hv[h] = (unsigned char)pv;
      }
    }
    if (j->payload >= 0) o->cols[j->payload].is_payload = 1;
  }
  for (int i = 0; i < o->ncols; ++i)
    if (o->cols[i].table == 0 && !o->cols[i].data) { snprintf(o->err, sizeof o->err, "column %s has no data", o->cols[i].name); rc = -1; goto done; }

  /* Scan. */
  {
    const long long N = o->rows[0];
    ScanState st;
    memset(&st, 0, sizeof st);
    st.o = o;
    st.result = result;
    st.validity = validity;
    st.G = G;
    st.ts = ts;
    st.vts = vts;
    for (int a = 0; a < o->naggs; ++a) st.acc[a] = o->aggs[a].fn == 2 ? ~0ULL : 0;
    st.touched = o->ngroups ? (unsigned char*)calloc(G, 1) : NULL;
    RowCtx rcx = {o, 0};
    for (long long r = 0; r < N; ++r) {
      rcx.row = r;
      walk(&st, &rcx, 0);
    }
    uint64_t* acc = st.acc;
    uint64_t* seen = st.seen;
    uint64_t* cnt = st.cnt;
    unsigned char* touched = st.touched;
    const long long derr = st.derr;
    if (o->ngroups == 0) {
      int avg_i = 0;
      for (int a = 0; a < o->naggs; ++a) {
        const AggS* ag = &o->aggs[a];
        if (ag->fn == 2) { if (acc[a] < result[a]) result[a] = acc[a]; }
        else if (ag->fn == 3) { if (acc[a] > result[a]) result[a] = acc[a]; }
        else result[a] += acc[a];
        if (ag->fn == 0 && N > 0) set_bit(validity, a);
        if ((ag->fn == 1 || ag->fn == 2 || ag->fn == 3) && seen[a]) set_bit(validity, a);
        if (ag->fn == 4) { result[vts + avg_i] += cnt[a]; avg_i++; }
      }
    } else {
      /* Key slots of every touched group (canonical values). */
      for (uint64_t g = 0; g < G; ++g) {
        if (!touched[g]) continue;
        long long rem = (long long)g;
        long long digit[16];
        for (int k = o->ngroups - 1; k >= 0; --k) {
          const long long card = o->groups[k].card + (o->groups[k].nullable ? 1 : 0);
          digit[k] = rem % card;
          rem /= card;
        }
        for (int k = 0; k < o->ngroups; ++k) {
          const GroupS* gs = &o->groups[k];
          const uint64_t slot = g * ts + k;
          if (gs->nullable && digit[k] == 0) { result[slot] = 0; continue; }
          result[slot] = (uint64_t)(digit[k] - (gs->nullable ? 1 : 0) + gs->min);
          if (!o->sparse) set_bit(validity, slot);
        }
      }
    }
    free(touched);
    if (domain_errors) *domain_errors = derr;
  }

  /* AVG finalisation: compacts storage tuples to visible tuples. */
  if (navg) {
    uint64_t* vr = (uint64_t*)calloc(G * vts + 1, 8);
    uint64_t* vv = (uint64_t*)calloc((G * vts + 63) / 64 + 1, 8);
    for (uint64_t g = 0; g < G; ++g) {
      const uint64_t src = g * ts, dst = g * vts;
      int slot = 0, avg_i = 0;
      for (int k = 0; k < o->ngroups; ++k, ++slot) {
        vr[dst + slot] = result[src + slot];
        if (get_bit(validity, src + slot)) set_bit(vv, dst + slot);
      }
      for (int a = 0; a < o->naggs; ++a, ++slot) {
        const AggS* ag = &o->aggs[a];
        if (ag->fn == 0) {
          vr[dst + slot] = result[src + slot];
          if (o->ngroups == 0 || result[src + slot] != 0) set_bit(vv, dst + slot);
        } else if (ag->fn == 4) {
          const uint64_t c = result[src + vts + avg_i];
          avg_i++;
          if (c) {
            double d = (double)result[src + slot] / (double)c;
            memcpy(&vr[dst + slot], &d, 8);
            set_bit(vv, dst + slot);
          }
        } else {
          vr[dst + slot] = (ag->fn == 2 && result[src + slot] == ~0ULL) ? 0 : result[src + slot];
          if (get_bit(validity, src + slot)) set_bit(vv, dst + slot);
        }
      }
    }
    memcpy(result, vr, G * vts * 8);
    memcpy(validity, vv, ((G * vts + 63) / 64) * 8);
    free(vr);
    free(vv);
  }

done:
  if (rc && err && errlen > 0) snprintf(err, (size_t)errlen, "%s", o->err);
  for (int s = 0; s < o->nsteps; ++s) {
    if (o->steps[s].kind == 0) free_expr(o->steps[s].filter);
    else {
      JoinS* j = &o->steps[s].join;
      free_expr(j->filter);
      free(j->ht);
      free(j->hv);
      free(j->mkey);
      free(j->mcnt);
      free(j->moff);
      free(j->mrows);
    }
  }
  for (int g = 0; g < o->ngroups; ++g) free_expr(o->groups[g].e);
  for (int a = 0; a < o->naggs; ++a) free_expr(o->aggs[a].arg);
  free(o->payload_val);
  free(o->payload_valid);
  free(o);
  return rc;
}
