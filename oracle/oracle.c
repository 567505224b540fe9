/*
 * oracle.c — CPU restatement of Sirius's INNER equi-hash-join, used ONLY as test infrastructure:
 * the parity checker of the tests, the reference of smoke(), and the timed CPU baseline of
 * bench.py. Nothing in the product links or calls it.
 *
 * Semantics restated (not code):
 *   - INNER = every (probe row, build row) pair with equal keys
 *     (src/op/sirius_physical_hash_join.cpp:1871-1874, cudf::inner_join);
 *   - compare_nulls_: plain `=` joins are UNEQUAL, so a NULL key never matches; only when every
 *     key is IS NOT DISTINCT FROM do NULLs match each other (:252-264);
 *   - duplicates on either side multiply (SQL multiset semantics; test
 *     test/cpp/integration/test_gpu_execution_join_nulls.cpp:42-58 pins NULLs + duplicates);
 *   - output row = (probe row id, build row id, probe payloads..., build payloads...), the column
 *     order of gather_join_output (:1326-1358); INNER needs no NULL padding (DONT_CHECK, :1319).
 *
 * Algorithm: a chained hash table (head[] / next[] row links, like DuckDB's CPU join hash table)
 * built in parallel with an atomic exchange on head[], then a parallel probe over contiguous probe
 * ranges into per-thread buffers, then a parallel copy that also gathers the payload columns.
 * The hash is a Fibonacci multiplicative hash, independent of the GPU table's mixer.
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAX_THREADS 256

typedef struct {
  const void* data;
  const uint32_t* validity; /* NULL = all valid */
  int64_t voff;
  int64_t n;
  int width; /* key: 4 or 8 */
} or_keys;

static inline int or_valid(const uint32_t* v, int64_t off, int64_t i) {
  if (!v) return 1;
  const int64_t b = off + i;
  return (v[b >> 5] >> (b & 31)) & 1u;
}

static inline int64_t or_key(const or_keys* k, int64_t i) {
  return k->width == 4 ? (int64_t)((const int32_t*)k->data)[i] : ((const int64_t*)k->data)[i];
}

static inline uint64_t or_hash(int64_t key, int shift) {
  return ((uint64_t)key * 0x9E3779B97F4A7C15ull) >> shift;
}

typedef struct {
  int32_t* head;        /* 2^bits heads, -1 = empty */
  int32_t* next;        /* per build row */
  int32_t null_head;    /* chain of NULL-key build rows (nulls equal) */
  int bits;
  const or_keys* b;
} or_table;

typedef struct {
  or_table* t;
  int64_t lo, hi;
  int nulls_equal;
  _Atomic int32_t* null_head;
} or_build_arg;

static void* or_build_worker(void* p) {
  or_build_arg* a = (or_build_arg*)p;
  or_table* t = a->t;
  _Atomic int32_t* head = (_Atomic int32_t*)t->head;
  const int shift = 64 - t->bits;
  for (int64_t i = a->lo; i < a->hi; ++i) {
    if (or_valid(t->b->validity, t->b->voff, i)) {
      const uint64_t h = t->bits ? or_hash(or_key(t->b, i), shift) : 0;
      t->next[i] = atomic_exchange_explicit(&head[h], (int32_t)i, memory_order_relaxed);
    } else if (a->nulls_equal) {
      t->next[i] = atomic_exchange_explicit(a->null_head, (int32_t)i, memory_order_relaxed);
    }
  }
  return NULL;
}

typedef struct {
  const or_table* t;
  const or_keys* p;
  int64_t lo, hi;
  int nulls_equal;
  int count_only;
  int64_t count;
  int32_t* prid; /* per-thread buffers (count_only == 0) */
  int32_t* brid;
  int64_t cap;
  int failed;
} or_probe_arg;

static int or_push(or_probe_arg* a, int32_t pr, int32_t br) {
  if (a->count >= a->cap) {
    int64_t nc = a->cap ? a->cap * 2 : 1024;
    int32_t* np = (int32_t*)realloc(a->prid, (size_t)nc * sizeof(int32_t));
    if (!np) return 0;
    a->prid = np;
    int32_t* nb = (int32_t*)realloc(a->brid, (size_t)nc * sizeof(int32_t));
    if (!nb) return 0;
    a->brid = nb;
    a->cap = nc;
  }
  a->prid[a->count] = pr;
  a->brid[a->count] = br;
  a->count++;
  return 1;
}

static void* or_probe_worker(void* p) {
  or_probe_arg* a = (or_probe_arg*)p;
  const or_table* t = a->t;
  const or_keys* b = t->b;
  const int shift = 64 - t->bits;
  for (int64_t i = a->lo; i < a->hi; ++i) {
    int32_t j;
    if (or_valid(a->p->validity, a->p->voff, i)) {
      const int64_t k = or_key(a->p, i);
      const uint64_t h = t->bits ? or_hash(k, shift) : 0;
      for (j = t->head[h]; j >= 0; j = t->next[j]) {
        if (or_key(b, j) != k) continue;
        if (a->count_only) a->count++;
        else if (!or_push(a, (int32_t)i, j)) { a->failed = 1; return NULL; }
      }
    } else if (a->nulls_equal) {
      for (j = t->null_head; j >= 0; j = t->next[j]) {
        if (a->count_only) a->count++;
        else if (!or_push(a, (int32_t)i, j)) { a->failed = 1; return NULL; }
      }
    }
  }
  return NULL;
}

typedef struct {
  const or_probe_arg* src;
  int64_t dst_off;
  int64_t capacity;
  int32_t* out_prid;
  int32_t* out_brid;
  int n_pp, n_bp;
  const void* const* pp;
  const int* pp_w;
  void* const* out_pp;
  const void* const* bp;
  const int* bp_w;
  void* const* out_bp;
} or_copy_arg;

static inline void or_copy_elem(void* dst, int64_t di, const void* src, int64_t si, int w) {
  memcpy((char*)dst + di * w, (const char*)src + si * w, (size_t)w);
}

static void* or_copy_worker(void* p) {
  or_copy_arg* a = (or_copy_arg*)p;
  const or_probe_arg* s = a->src;
  for (int64_t r = 0; r < s->count; ++r) {
    const int64_t d = a->dst_off + r;
    if (d >= a->capacity) break;
    const int32_t pr = s->prid[r], br = s->brid[r];
    if (a->out_prid) a->out_prid[d] = pr;
    if (a->out_brid) a->out_brid[d] = br;
    for (int c = 0; c < a->n_pp; ++c) or_copy_elem(a->out_pp[c], d, a->pp[c], pr, a->pp_w[c]);
    for (int c = 0; c < a->n_bp; ++c) or_copy_elem(a->out_bp[c], d, a->bp[c], br, a->bp_w[c]);
  }
  return NULL;
}

static int or_threads(int threads, int64_t work) {
  if (threads < 1) threads = 1;
  if (threads > OR_MAX_THREADS) threads = OR_MAX_THREADS;
  if (work < (int64_t)threads * 4096) {
    int64_t t = work / 4096;
    threads = t < 1 ? 1 : (int)t;
  }
  return threads;
}

static int or_build(or_table* t, const or_keys* b, int nulls_equal, int threads) {
  int bits = 1;
  while (((int64_t)1 << bits) < 2 * (b->n > 0 ? b->n : 1)) ++bits;
  t->bits = bits;
  t->b = b;
  t->null_head = -1;
  t->head = (int32_t*)malloc(((size_t)1 << bits) * sizeof(int32_t));
  t->next = (int32_t*)malloc((size_t)(b->n > 0 ? b->n : 1) * sizeof(int32_t));
  if (!t->head || !t->next) return 0;
  memset(t->head, 0xff, ((size_t)1 << bits) * sizeof(int32_t));
  const int nt = or_threads(threads, b->n);
  pthread_t th[OR_MAX_THREADS];
  or_build_arg args[OR_MAX_THREADS];
  _Atomic int32_t null_head = -1;
  for (int i = 0; i < nt; ++i) {
    args[i].t = t;
    args[i].lo = b->n * i / nt;
    args[i].hi = b->n * (i + 1) / nt;
    args[i].nulls_equal = nulls_equal;
    args[i].null_head = &null_head;
    if (nt > 1) pthread_create(&th[i], NULL, or_build_worker, &args[i]);
    else or_build_worker(&args[i]);
  }
  if (nt > 1)
    for (int i = 0; i < nt; ++i) pthread_join(th[i], NULL);
  t->null_head = atomic_load(&null_head);
  return 1;
}

static void or_free(or_table* t) {
  free(t->head);
  free(t->next);
}

/* Number of INNER matches. Returns -1 on allocation failure. */
int64_t oracle_join_count(const void* bkeys, const uint32_t* bvalid, int64_t bvoff, int64_t nb,
                          const void* pkeys, const uint32_t* pvalid, int64_t pvoff, int64_t np,
                          int key_width, int nulls_equal, int threads) {
  or_keys b = {bkeys, bvalid, bvoff, nb, key_width};
  or_keys p = {pkeys, pvalid, pvoff, np, key_width};
  or_table t;
  if (!or_build(&t, &b, nulls_equal, threads)) { or_free(&t); return -1; }
  const int nt = or_threads(threads, np);
  pthread_t th[OR_MAX_THREADS];
  or_probe_arg args[OR_MAX_THREADS];
  memset(args, 0, sizeof(args));
  for (int i = 0; i < nt; ++i) {
    args[i].t = &t;
    args[i].p = &p;
    args[i].lo = np * i / nt;
    args[i].hi = np * (i + 1) / nt;
    args[i].nulls_equal = nulls_equal;
    args[i].count_only = 1;
    if (nt > 1) pthread_create(&th[i], NULL, or_probe_worker, &args[i]);
    else or_probe_worker(&args[i]);
  }
  int64_t total = 0;
  for (int i = 0; i < nt; ++i) {
    if (nt > 1) pthread_join(th[i], NULL);
    total += args[i].count;
  }
  or_free(&t);
  return total;
}

/* INNER join with the payload gather. Writes min(M, capacity) rows in probe-row order and returns
 * M (the total number of matches), or -1 on allocation failure. Any out pointer may be NULL when
 * capacity is 0; out_prid / out_brid may be NULL to skip them. */
int64_t oracle_inner_join(const void* bkeys, const uint32_t* bvalid, int64_t bvoff, int64_t nb,
                          const void* pkeys, const uint32_t* pvalid, int64_t pvoff, int64_t np,
                          int key_width, int nulls_equal, int threads,
                          int32_t* out_prid, int32_t* out_brid, int64_t capacity,
                          int n_pp, const void* const* pp, const int* pp_w, void* const* out_pp,
                          int n_bp, const void* const* bp, const int* bp_w, void* const* out_bp) {
  or_keys b = {bkeys, bvalid, bvoff, nb, key_width};
  or_keys p = {pkeys, pvalid, pvoff, np, key_width};
  or_table t;
  if (!or_build(&t, &b, nulls_equal, threads)) { or_free(&t); return -1; }
  const int nt = or_threads(threads, np);
  pthread_t th[OR_MAX_THREADS];
  or_probe_arg args[OR_MAX_THREADS];
  memset(args, 0, sizeof(args));
  for (int i = 0; i < nt; ++i) {
    args[i].t = &t;
    args[i].p = &p;
    args[i].lo = np * i / nt;
    args[i].hi = np * (i + 1) / nt;
    args[i].nulls_equal = nulls_equal;
    if (nt > 1) pthread_create(&th[i], NULL, or_probe_worker, &args[i]);
    else or_probe_worker(&args[i]);
  }
  int64_t total = 0;
  int failed = 0;
  or_copy_arg cargs[OR_MAX_THREADS];
  for (int i = 0; i < nt; ++i) {
    if (nt > 1) pthread_join(th[i], NULL);
    failed |= args[i].failed;
    cargs[i].src = &args[i];
    cargs[i].dst_off = total;
    cargs[i].capacity = capacity;
    cargs[i].out_prid = out_prid;
    cargs[i].out_brid = out_brid;
    cargs[i].n_pp = n_pp;
    cargs[i].pp = pp;
    cargs[i].pp_w = pp_w;
    cargs[i].out_pp = out_pp;
    cargs[i].n_bp = n_bp;
    cargs[i].bp = bp;
    cargs[i].bp_w = bp_w;
    cargs[i].out_bp = out_bp;
    total += args[i].count;
  }
  if (!failed) {
    for (int i = 0; i < nt; ++i) {
      if (nt > 1) pthread_create(&th[i], NULL, or_copy_worker, &cargs[i]);
      else or_copy_worker(&cargs[i]);
    }
    if (nt > 1)
      for (int i = 0; i < nt; ++i) pthread_join(th[i], NULL);
  }
  for (int i = 0; i < nt; ++i) {
    free(args[i].prid);
    free(args[i].brid);
  }
  or_free(&t);
  return failed ? -1 : total;
}
