/*
 * tree_oracle.c -- CPU restatement of the reference TreeDeduplicator (tree approach,
 * low-offset first occurrence) used ONLY as the correctness checker.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * / reference arm may load this library.  The product (libb200dedup.so) never links,
 * loads or calls it, and has no CPU fallback.
 *
 * Every function follows the reference source in execution order as if the Kokkos
 * dispatches ran sequentially (one thread, ascending index), which is the canonical
 * output order the GPU library must reproduce:
 *   chunk hash ........ include/hash_functions.hpp:16-20 -> include/kokkos_murmur3.hpp:213-292
 *                       (rotl64 returns uint32_t, kokkos_murmur3.hpp:30-31; seed 0, :436)
 *                       or include/kokkos_md5.hpp:287-323 (standard MD5, RFC 1321)
 *   tree index math ... include/kokkos_merkle_tree.hpp:102-142
 *   baseline dedup .... src/tree_approach.cpp:13-259
 *   incremental dedup . src/tree_approach.cpp:261-509
 *   diff assembly ..... src/tree_approach.cpp:511-710
 *   checkpoint ........ src/tree_approach.cpp:1577-1689
 *   host-view restart . src/tree_approach.cpp:712-1128
 * The only deviation: the chunk digests of one checkpoint are computed up front
 * (optionally with OpenMP threads).  Hashing is a pure function of the chunk bytes,
 * so this changes no result; every map insert and label decision stays sequential.
 *
 * Memory safety: where the reference would index outside a buffer (only reachable with
 * corrupt diffs or the non-power-of-two region-size quirk), the oracle skips the access
 * and reports ORACLE_WARN_OOB instead of reading or writing out of bounds.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_OK 0
#define ORACLE_ERR_ARG (-1)
#define ORACLE_ERR_NOMEM (-2)
#define ORACLE_ERR_FORMAT (-3)
#define ORACLE_WARN_OOB 2

enum { HASH_MURMUR3 = 0, HASH_MD5 = 1 };
/* include/utils.hpp:51-57 */
enum { FIRST_OCUR = 0, FIXED_DUPL = 1, SHIFT_DUPL = 2, FIRST_DUPL = 3, DONE = 4 };

typedef struct { uint8_t b[16]; } digest_t;            /* include/map_helpers.hpp:7-9 */
typedef struct { uint32_t node, tree; } nodeid_t;     /* include/map_helpers.hpp:38-58 */

/* ------------------------------------------------------------------------------------ */
/* Murmur3 x64-128 as the reference computes it: every 64-bit rotate is truncated to its */
/* low 32 bits because rotl64 is declared to return uint32_t (kokkos_murmur3.hpp:30-31). */
/* ------------------------------------------------------------------------------------ */
static inline uint64_t rotl_trunc(uint64_t x, int r) {
  return (uint32_t)((x << r) | (x >> (64 - r)));
}
static inline uint64_t fmix64(uint64_t k) {            /* kokkos_murmur3.hpp:44-53 */
  k ^= k >> 33; k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33; return k;
}
static inline uint64_t ld64(const uint8_t* p) { uint64_t v; memcpy(&v, p, 8); return v; }

void oracle_murmur3(const uint8_t* data, uint64_t len, uint8_t out[16]) {
  /* kokkos_murmur3.hpp:213-292 with seed 0 (:436) */
  const uint64_t c1 = 0x87c37b91114253d5ULL, c2 = 0x4cf5ad432745937fULL;
  uint64_t h1 = 0, h2 = 0, nblocks = len / 16;
  for (uint64_t i = 0; i < nblocks; i++) {
    uint64_t k1 = ld64(data + 16 * i), k2 = ld64(data + 16 * i + 8);
    k1 *= c1; k1 = rotl_trunc(k1, 31); k1 *= c2; h1 ^= k1;
    h1 = rotl_trunc(h1, 27); h1 += h2; h1 = h1 * 5 + 0x52dce729;
    k2 *= c2; k2 = rotl_trunc(k2, 33); k2 *= c1; h2 ^= k2;
    h2 = rotl_trunc(h2, 31); h2 += h1; h2 = h2 * 5 + 0x38495ab5;
  }
  const uint8_t* tail = data + nblocks * 16;
  uint64_t k1 = 0, k2 = 0;
  unsigned rem = (unsigned)(len & 15);
  if (rem > 8) {
    for (unsigned i = rem; i > 8; i--) k2 ^= ((uint64_t)tail[i - 1]) << (8 * (i - 9));
    k2 *= c2; k2 = rotl_trunc(k2, 33); k2 *= c1; h2 ^= k2;
  }
  if (rem > 0) {
    unsigned top = rem > 8 ? 8 : rem;
    for (unsigned i = top; i > 0; i--) k1 ^= ((uint64_t)tail[i - 1]) << (8 * (i - 1));
    k1 *= c1; k1 = rotl_trunc(k1, 31); k1 *= c2; h1 ^= k1;
  }
  h1 ^= len; h2 ^= len;
  h1 += h2; h2 += h1;
  h1 = fmix64(h1); h2 = fmix64(h2);
  h1 += h2; h2 += h1;
  memcpy(out, &h1, 8); memcpy(out + 8, &h2, 8);
}

/* ------------------------------------------------------------------------------------ */
/* MD5 (RFC 1321).  kokkos_md5.hpp:287-323 is a standard MD5; the round constants are   */
/* floor(2^32 * |sin(i+1)|), tabulated here as in the RFC.                              */
/* ------------------------------------------------------------------------------------ */
static const uint32_t MD5_T[64] = {
  0xd76aa478,0xe8c7b756,0x242070db,0xc1bdceee,0xf57c0faf,0x4787c62a,0xa8304613,0xfd469501,
  0x698098d8,0x8b44f7af,0xffff5bb1,0x895cd7be,0x6b901122,0xfd987193,0xa679438e,0x49b40821,
  0xf61e2562,0xc040b340,0x265e5a51,0xe9b6c7aa,0xd62f105d,0x02441453,0xd8a1e681,0xe7d3fbc8,
  0x21e1cde6,0xc33707d6,0xf4d50d87,0x455a14ed,0xa9e3e905,0xfcefa3f8,0x676f02d9,0x8d2a4c8a,
  0xfffa3942,0x8771f681,0x6d9d6122,0xfde5380c,0xa4beea44,0x4bdecfa9,0xf6bb4b60,0xbebfbc70,
  0x289b7ec6,0xeaa127fa,0xd4ef3085,0x04881d05,0xd9d4d039,0xe6db99e5,0x1fa27cf8,0xc4ac5665,
  0xf4292244,0x432aff97,0xab9423a7,0xfc93a039,0x655b59c3,0x8f0ccc92,0xffeff47d,0x85845dd1,
  0x6fa87e4f,0xfe2ce6e0,0xa3014314,0x4e0811a1,0xf7537e82,0xbd3af235,0x2ad7d2bb,0xeb86d391};
static const uint8_t MD5_S[64] = {
  7,12,17,22,7,12,17,22,7,12,17,22,7,12,17,22, 5,9,14,20,5,9,14,20,5,9,14,20,5,9,14,20,
  4,11,16,23,4,11,16,23,4,11,16,23,4,11,16,23, 6,10,15,21,6,10,15,21,6,10,15,21,6,10,15,21};

static void md5_block(uint32_t st[4], const uint8_t blk[64]) {
  uint32_t m[16];
  for (int i = 0; i < 16; i++)
    m[i] = (uint32_t)blk[4*i] | ((uint32_t)blk[4*i+1] << 8) | ((uint32_t)blk[4*i+2] << 16) |
           ((uint32_t)blk[4*i+3] << 24);
  uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
  for (int i = 0; i < 64; i++) {
    uint32_t f; int g;
    if (i < 16)      { f = (b & c) | (~b & d); g = i; }
    else if (i < 32) { f = (d & b) | (~d & c); g = (5 * i + 1) & 15; }
    else if (i < 48) { f = b ^ c ^ d;          g = (3 * i + 5) & 15; }
    else             { f = c ^ (b | ~d);       g = (7 * i) & 15; }
    uint32_t t = a + f + MD5_T[i] + m[g];
    a = d; d = c; c = b;
    b = b + ((t << MD5_S[i]) | (t >> (32 - MD5_S[i])));
  }
  st[0] += a; st[1] += b; st[2] += c; st[3] += d;
}

void oracle_md5(const uint8_t* data, uint64_t len, uint8_t out[16]) {
  uint32_t st[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
  uint64_t full = len / 64;
  for (uint64_t i = 0; i < full; i++) md5_block(st, data + 64 * i);
  uint8_t buf[128];
  unsigned rem = (unsigned)(len - full * 64);
  memset(buf, 0, sizeof buf);
  memcpy(buf, data + full * 64, rem);
  buf[rem] = 0x80;
  unsigned tot = (rem < 56) ? 64 : 128;
  uint64_t bits = len * 8;
  for (int i = 0; i < 8; i++) buf[tot - 8 + i] = (uint8_t)(bits >> (8 * i));
  md5_block(st, buf);
  if (tot == 128) md5_block(st, buf + 64);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) out[4 * i + j] = (uint8_t)(st[i] >> (8 * j));
}

void oracle_hash(int kind, const uint8_t* data, uint64_t len, uint8_t out[16]) {
  if (kind == HASH_MD5) oracle_md5(data, len, out); else oracle_murmur3(data, len, out);
}

/* ------------------------------------------------------------------------------------ */
/* Tree index math: include/kokkos_merkle_tree.hpp:102-142, restated as one helper that  */
/* returns both ends (the reference repeats the same loop in three functions).           */
/* ------------------------------------------------------------------------------------ */
static void leaf_range(uint32_t node, uint32_t num_nodes, uint32_t* lo, uint32_t* hi) {
  uint32_t l = 2 * node + 1, r = 2 * node + 2;
  while (l < num_nodes) { l = 2 * l + 1; r = 2 * r + 2; }
  l = (l - 1) / 2; r = (r - 2) / 2;
  if (r > num_nodes) r = num_nodes - 1;
  *lo = l; *hi = r;
}
uint32_t oracle_num_leaf_descendents(uint32_t node, uint32_t num_nodes) {
  uint32_t l, r; leaf_range(node, num_nodes, &l, &r); return r - l + 1;
}
uint32_t oracle_leftmost_leaf(uint32_t node, uint32_t num_nodes) {
  uint32_t l, r; leaf_range(node, num_nodes, &l, &r); return l;
}

/* ------------------------------------------------------------------------------------ */
/* Sequential digest -> NodeID map with the UnorderedMap insert contract used by the     */
/* tree path (include/map_helpers.hpp:60-113): insert-if-absent, reporting success or    */
/* existing plus the slot index; value_at(index) is mutable.                              */
/* ------------------------------------------------------------------------------------ */
typedef struct {
  digest_t* keys;
  nodeid_t* vals;
  uint8_t* used;
  uint64_t cap, size;
} dmap_t;

static uint64_t dmap_slot(const digest_t* k, uint64_t cap) {
  uint64_t a, b; memcpy(&a, k->b, 8); memcpy(&b, k->b + 8, 8);
  uint64_t h = (a ^ (b * 0x9E3779B97F4A7C15ULL)); h ^= h >> 29;
  return h % cap;
}
static int dmap_init(dmap_t* m, uint64_t cap) {
  memset(m, 0, sizeof *m);
  if (cap < 16) cap = 16;
  m->keys = (digest_t*)malloc(cap * sizeof(digest_t));
  m->vals = (nodeid_t*)malloc(cap * sizeof(nodeid_t));
  m->used = (uint8_t*)calloc(cap, 1);
  if (!m->keys || !m->vals || !m->used) return ORACLE_ERR_NOMEM;
  m->cap = cap;
  return ORACLE_OK;
}
static void dmap_free(dmap_t* m) { free(m->keys); free(m->vals); free(m->used); memset(m, 0, sizeof *m); }
static int64_t dmap_find(const dmap_t* m, const digest_t* k) {
  uint64_t s = dmap_slot(k, m->cap);
  while (m->used[s]) {
    if (memcmp(m->keys[s].b, k->b, 16) == 0) return (int64_t)s;
    if (++s == m->cap) s = 0;
  }
  return -1;
}
/* returns slot; *inserted = 1 on success, 0 when the key already existed */
static int64_t dmap_insert_raw(dmap_t* m, const digest_t* k, nodeid_t v, int* inserted) {
  uint64_t s = dmap_slot(k, m->cap);
  while (m->used[s]) {
    if (memcmp(m->keys[s].b, k->b, 16) == 0) { *inserted = 0; return (int64_t)s; }
    if (++s == m->cap) s = 0;
  }
  m->used[s] = 1; m->keys[s] = *k; m->vals[s] = v; m->size++;
  *inserted = 1;
  return (int64_t)s;
}
static int dmap_rehash(dmap_t* m, uint64_t want) {
  /* capacity policy is internal; keep load <= 1/2 so probing stays short */
  if (2 * want + 16 <= m->cap) return ORACLE_OK;
  uint64_t cap = 3 * want + 16;
  dmap_t n;
  if (dmap_init(&n, cap)) return ORACLE_ERR_NOMEM;
  for (uint64_t s = 0; s < m->cap; s++)
    if (m->used[s]) { int ins; dmap_insert_raw(&n, &m->keys[s], m->vals[s], &ins); }
  dmap_free(m);
  *m = n;
  return ORACLE_OK;
}
static int64_t dmap_insert(dmap_t* m, const digest_t* k, nodeid_t v, int* inserted) {
  if (2 * (m->size + 1) > m->cap && dmap_rehash(m, m->size + 1)) { *inserted = -1; return -1; }
  return dmap_insert_raw(m, k, v, inserted);
}

/* ------------------------------------------------------------------------------------ */
/* Deduplicator state: include/tree_approach.hpp:16-59                                    */
/* ------------------------------------------------------------------------------------ */
typedef struct {
  uint32_t* v; uint64_t n, cap;
} u32vec_t;
static int vec_push(u32vec_t* v, uint32_t x) {
  if (v->n == v->cap) {
    uint64_t c = v->cap ? 2 * v->cap : 64;
    uint32_t* p = (uint32_t*)realloc(v->v, c * sizeof(uint32_t));
    if (!p) return ORACLE_ERR_NOMEM;
    v->v = p; v->cap = c;
  }
  v->v[v->n++] = x;
  return ORACLE_OK;
}

typedef struct oracle_dedup {
  uint32_t chunk_size;
  int hash_kind;
  int threads;
  uint32_t current_id, baseline_id;
  uint64_t data_len;
  uint32_t num_chunks, num_nodes;
  digest_t* tree; uint64_t tree_nodes;
  dmap_t map; int map_ready;
  u32vec_t first_vec, shift_vec;
  uint8_t* labels;           /* last checkpoint's labels, kept for inspection */
  uint64_t datasizes[2];
} oracle_dedup;

oracle_dedup* oracle_create(uint32_t chunk_size, int hash_kind) {
  if (chunk_size == 0) return NULL;
  oracle_dedup* d = (oracle_dedup*)calloc(1, sizeof(oracle_dedup));
  if (!d) return NULL;
  d->chunk_size = chunk_size;          /* src/tree_approach.cpp:5-9 */
  d->hash_kind = hash_kind;
  d->threads = 1;
  return d;
}
void oracle_destroy(oracle_dedup* d) {
  if (!d) return;
  free(d->tree); dmap_free(&d->map); free(d->first_vec.v); free(d->shift_vec.v); free(d->labels);
  free(d);
}
void oracle_set_threads(oracle_dedup* d, int t) { d->threads = t < 1 ? 1 : t; }
uint64_t oracle_num_first_ocur(const oracle_dedup* d) { return d->first_vec.n; }
uint64_t oracle_num_shift_dupl(const oracle_dedup* d) { return d->shift_vec.n; }
uint32_t oracle_current_id(const oracle_dedup* d) { return d->current_id; }
void oracle_datasizes(const oracle_dedup* d, uint64_t out[2]) { out[0] = d->datasizes[0]; out[1] = d->datasizes[1]; }
const uint8_t* oracle_tree(const oracle_dedup* d, uint64_t* nnodes) { *nnodes = d->tree_nodes; return (const uint8_t*)d->tree; }
const uint8_t* oracle_labels(const oracle_dedup* d) { return d->labels; }
const uint32_t* oracle_first_list(const oracle_dedup* d) { return d->first_vec.v; }
const uint32_t* oracle_shift_list(const oracle_dedup* d) { return d->shift_vec.v; }
int oracle_map_lookup(const oracle_dedup* d, const uint8_t key[16], uint32_t out[2]) {
  digest_t k; memcpy(k.b, key, 16);
  int64_t s = dmap_find(&d->map, &k);
  if (s < 0) return 0;
  out[0] = d->map.vals[s].node; out[1] = d->map.vals[s].tree;
  return 1;
}
uint64_t oracle_map_size(const oracle_dedup* d) { return d->map.size; }

static void hash_pair(int kind, const digest_t* l, digest_t* out) {
  /* inner nodes hash 32 bytes: left child digest then right (tree_approach.cpp:131,221,389,459) */
  oracle_hash(kind, (const uint8_t*)l, 2 * sizeof(digest_t), out->b);
}

static void hash_leaves(oracle_dedup* d, const uint8_t* data, uint64_t len, digest_t* dig) {
  const uint32_t n = d->num_chunks;
  const uint64_t cs = d->chunk_size;
  const int kind = d->hash_kind;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(d->threads)
#endif
  for (int64_t c = 0; c < (int64_t)n; c++) {
    uint64_t off = (uint64_t)c * cs;
    uint64_t nb = (c == (int64_t)n - 1) ? len - off : cs;   /* :319-320 */
    oracle_hash(kind, data + off, nb, dig[c].b);
  }
}

/* level iteration: start at the deepest level (tree_approach.cpp:42-48) and walk up */
#define FOR_LEVELS_BOTTOM_UP(beg, end, N)                                   \
  for (beg = 0, end = 0; end < (N); beg = 2 * beg + 1, end = 2 * end + 2) {} \
  for (; beg <= (N); beg = (beg - 1) / 2, end = (end - 2) / 2)

static int push_child(oracle_dedup* d, const uint8_t* labels, uint32_t child) {
  if (labels[child] != FIXED_DUPL && labels[child] != DONE) {
    if (labels[child] == SHIFT_DUPL) return vec_push(&d->shift_vec, child);
    return vec_push(&d->first_vec, child);
  }
  return ORACLE_OK;
}

/* src/tree_approach.cpp:13-259 (baseline) and :261-509 (incremental) */
static int dedup(oracle_dedup* d, const uint8_t* data, uint64_t len, int baseline) {
  const uint32_t n = d->num_chunks, N = d->num_nodes, cur = d->current_id;
  const int kind = d->hash_kind;
  digest_t* dig = (digest_t*)malloc((uint64_t)n * sizeof(digest_t));
  uint8_t* labels = (uint8_t*)malloc(N);
  if (!dig || !labels) { free(dig); free(labels); return ORACLE_ERR_NOMEM; }
  memset(labels, DONE, N);
  hash_leaves(d, data, len, dig);
  dmap_t* m = &d->map;
  digest_t* tree = d->tree;
  int rc = ORACLE_OK;

  /* Leaves (:54-94 baseline, :305-351 incremental) */
  for (uint32_t leaf = n - 1; leaf < N; leaf++) {
    digest_t* dg = &dig[leaf - (n - 1)];
    int ins;
    int64_t s = dmap_insert(m, dg, (nodeid_t){leaf, cur}, &ins);
    if (ins < 0) { rc = ORACLE_ERR_NOMEM; goto out; }
    if (memcmp(dg->b, tree[leaf].b, 16) == 0) {
      labels[leaf] = FIXED_DUPL;
      if (baseline) tree[leaf] = *dg;
    } else if (ins) {
      labels[leaf] = FIRST_OCUR;
      tree[leaf] = *dg;
    } else {
      nodeid_t* info = &m->vals[s];
      if (info->tree == cur) {
        if (leaf < info->node) info->node = leaf;   /* atomic_min */
        labels[leaf] = FIRST_OCUR;
      } else {
        labels[leaf] = SHIFT_DUPL;
      }
      tree[leaf] = *dg;
    }
  }
  /* Choose first occurrences (:100-114, :353-369) */
  for (uint32_t leaf = n - 1; leaf < N; leaf++) {
    if (labels[leaf] == FIRST_OCUR) {
      int64_t s = dmap_find(m, &tree[leaf]);
      nodeid_t info = m->vals[s];
      if (info.tree == cur && leaf != info.node) labels[leaf] = SHIFT_DUPL;
    }
  }
  uint32_t beg, end;
  /* First occurrence forest (:116-145, :371-404) */
  FOR_LEVELS_BOTTOM_UP(beg, end, N) {
    for (uint64_t node = beg; node <= end; node++) {
      if (node < (uint64_t)n - 1) {
        uint32_t l = 2 * (uint32_t)node + 1, r = 2 * (uint32_t)node + 2;
        if (labels[l] == FIRST_OCUR && labels[r] == FIRST_OCUR) {
          labels[node] = FIRST_OCUR;
          hash_pair(kind, &tree[l], &tree[node]);
          int ins;
          dmap_insert(m, &tree[node], (nodeid_t){(uint32_t)node, cur}, &ins);
          if (ins < 0) { rc = ORACLE_ERR_NOMEM; goto out; }
        }
        if (node == 0 && labels[0] == FIRST_OCUR)
          if ((rc = vec_push(&d->first_vec, 0))) goto out;
      }
    }
  }
  /* Forest of region roots (:147-224 baseline, :406-477 incremental) */
  FOR_LEVELS_BOTTOM_UP(beg, end, N) {
    for (uint64_t node = beg; node <= end; node++) {
      if (node >= (uint64_t)n - 1) continue;
      uint32_t l = 2 * (uint32_t)node + 1, r = 2 * (uint32_t)node + 2;
      if (labels[l] != labels[r]) {
        labels[node] = DONE;
        if ((rc = push_child(d, labels, l))) goto out;
        if ((rc = push_child(d, labels, r))) goto out;
      } else if (labels[l] == FIXED_DUPL) {
        labels[node] = FIXED_DUPL;
      } else if (labels[l] == SHIFT_DUPL) {
        /* baseline tests the digest before it is computed (:202); incremental hashes first (:459) */
        if (!baseline) hash_pair(kind, &tree[l], &tree[node]);
        if (dmap_find(m, &tree[node]) >= 0) {
          labels[node] = SHIFT_DUPL;
        } else {
          labels[node] = DONE;
          if ((rc = vec_push(&d->shift_vec, l))) goto out;
          if ((rc = vec_push(&d->shift_vec, r))) goto out;
        }
      }
    }
    if (baseline) {   /* "Baseline: Build Forest: Insert entries" (:218-224) */
      for (uint64_t node = beg; node <= end; node++) {
        if (node >= (uint64_t)n - 1) continue;
        uint32_t l = 2 * (uint32_t)node + 1;
        hash_pair(kind, &tree[l], &tree[node]);
        int ins;
        dmap_insert(m, &tree[node], (nodeid_t){(uint32_t)node, cur}, &ins);
        if (ins < 0) { rc = ORACLE_ERR_NOMEM; goto out; }
      }
    }
  }
out:
  free(dig);
  free(d->labels);
  d->labels = labels;
  return rc;
}

/* src/tree_approach.cpp:511-710 */
static int collect_diff(oracle_dedup* d, const uint8_t* data, uint64_t len,
                        uint8_t** out, uint64_t* out_len) {
  const uint32_t n = d->num_chunks, N = d->num_nodes, cur = d->current_id;
  const uint64_t cs = d->chunk_size;
  dmap_t* m = &d->map;
  const uint64_t F = d->first_vec.n, S = d->shift_vec.n;
  uint32_t* region_nodes = (uint32_t*)malloc((F + 1) * sizeof(uint32_t));
  uint32_t* region_off = (uint32_t*)malloc((F + 1) * sizeof(uint32_t));
  uint64_t* prior = (uint64_t*)calloc((uint64_t)cur + 1, sizeof(uint64_t));
  uint32_t* skey = (uint32_t*)malloc((S + 1) * sizeof(uint32_t));
  uint32_t* sprev = (uint32_t*)malloc((S + 1) * sizeof(uint32_t));
  uint8_t* buf = NULL;
  int rc = ORACLE_OK;
  if (!region_nodes || !region_off || !prior || !skey || !sprev) { rc = ORACLE_ERR_NOMEM; goto done; }
  /* Count first ocur bytes (:545-558) */
  uint32_t num_distinct = 0;
  uint64_t chunk_counter = 0;
  for (uint64_t i = 0; i < F; i++) {
    uint32_t node = d->first_vec.v[i];
    int64_t s = dmap_find(m, &d->tree[node]);
    nodeid_t prev = s >= 0 ? m->vals[s] : (nodeid_t){UINT32_MAX, UINT32_MAX};
    if (node == prev.node && cur == prev.tree) {
      uint32_t size = oracle_num_leaf_descendents(node, N);
      region_nodes[num_distinct] = node;
      region_off[num_distinct] = size;
      num_distinct++;
      chunk_counter += size;
    } else {
      fprintf(stderr, "oracle: distinct node with different node/tree\n");
    }
  }
  /* Count shift dupl bytes (:565-589) */
  for (uint64_t i = 0; i < S; i++) {
    uint32_t node = d->shift_vec.v[i];
    int64_t s = dmap_find(m, &d->tree[node]);
    nodeid_t prev = m->vals[s];
    prior[prev.tree] += 1;
    skey[i] = prev.tree;
    sprev[i] = prev.node;
  }
  uint32_t num_prior = 0;
  for (uint64_t t = 0; t <= cur; t++) num_prior += prior[t] > 0;
  /* Calculate offsets (:601-606): exclusive scan */
  uint32_t run = 0;
  for (uint32_t i = 0; i < num_distinct; i++) { uint32_t l = region_off[i]; region_off[i] = run; run += l; }
  /* Allocate buffer (:620-623) */
  uint64_t data_offset = F * 4 + S * 8 + (uint64_t)num_prior * 8;
  uint64_t buffer_len = 32 + F * 4 + 8 * (uint64_t)num_prior + S * 8 + chunk_counter * cs;
  buf = (uint8_t*)calloc(buffer_len ? buffer_len : 1, 1);
  if (!buf) { rc = ORACLE_ERR_NOMEM; goto done; }
  /* Copy first ocur metadata (:629-633) */
  for (uint32_t i = 0; i < num_distinct; i++) memcpy(buf + 32 + 4 * (uint64_t)i, &region_nodes[i], 4);
  /* Find region leaves + Copy data (:608-617, :635-650) */
  for (uint32_t i = 0; i < num_distinct; i++) {
    uint32_t node = region_nodes[i];
    uint32_t size = oracle_num_leaf_descendents(node, N);
    uint32_t start = oracle_leftmost_leaf(node, N) - (n - 1);
    for (uint32_t j = 0; j < size; j++) {
      uint32_t chunk = start + j;
      uint64_t k = (uint64_t)region_off[i] + j;
      uint64_t src = (uint64_t)chunk * cs;
      uint64_t wsz = cs;
      if (chunk == n - 1) wsz = len - src;
      uint64_t dst = 32 + data_offset + k * cs;
      if (src + wsz > len || dst + wsz > buffer_len || chunk >= n) { rc = ORACLE_WARN_OOB; continue; }
      memcpy(buf + dst, data + src, wsz);
    }
  }
  /* Write repeat count (:656-665): atomic cursor -> ascending checkpoint id sequentially */
  uint64_t pos = 4 * (uint64_t)num_distinct;
  for (uint32_t t = 0; t <= cur; t++) {
    if (prior[t] > 0) {
      uint32_t c = (uint32_t)prior[t];
      memcpy(buf + 32 + pos, &t, 4); memcpy(buf + 32 + pos + 4, &c, 4);
      pos += 8;
    }
  }
  /* BinSort by source checkpoint (:670-687), stable; Write repeat metadata (:690-696) */
  uint64_t prior_start = (uint64_t)num_distinct * 4 + (uint64_t)num_prior * 8;
  uint64_t w = 0;
  for (uint32_t t = 0; t <= cur; t++) {
    if (!prior[t]) continue;
    for (uint64_t i = 0; i < S; i++) {
      if (skey[i] != t) continue;
      memcpy(buf + 32 + prior_start + 8 * w, &d->shift_vec.v[i], 4);
      memcpy(buf + 32 + prior_start + 8 * w + 4, &sprev[i], 4);
      w++;
    }
  }
  /* header (:700-706) copied in on the host (:1684); include/utils.hpp:29-37 */
  {
    uint32_t h32;
    h32 = d->baseline_id; memcpy(buf + 0, &h32, 4);
    h32 = cur;            memcpy(buf + 4, &h32, 4);
    memcpy(buf + 8, &len, 8);
    h32 = d->chunk_size;  memcpy(buf + 16, &h32, 4);
    h32 = (uint32_t)F;    memcpy(buf + 20, &h32, 4);
    h32 = num_prior;      memcpy(buf + 24, &h32, 4);
    h32 = (uint32_t)S;    memcpy(buf + 28, &h32, 4);
  }
  {
    uint64_t size_metadata = F * 4 + (uint64_t)num_prior * 8 + S * 8;
    d->datasizes[0] = buffer_len - size_metadata;
    d->datasizes[1] = size_metadata;
  }
  *out = buf; *out_len = buffer_len; buf = NULL;
done:
  free(region_nodes); free(region_off); free(prior); free(skey); free(sprev); free(buf);
  return rc;
}

/* src/tree_approach.cpp:1577-1689 plus the current_id += 1 of the host-view overload :1740-1748 */
int oracle_checkpoint(oracle_dedup* d, const uint8_t* data, uint64_t len, int make_baseline,
                      uint8_t** diff, uint64_t* diff_len) {
  if (!d || !diff || !diff_len || len == 0) return ORACLE_ERR_ARG;
  uint64_t nc = len / d->chunk_size;
  if (nc * d->chunk_size < len) nc += 1;
  if (nc > 0x7fffffffULL) return ORACLE_ERR_ARG;
  d->data_len = len;
  d->num_chunks = (uint32_t)nc;
  d->num_nodes = 2 * d->num_chunks - 1;
  int baseline = (d->current_id == 0) || make_baseline;
  if (make_baseline || !d->tree) {
    if (make_baseline || !d->map_ready) {
      dmap_free(&d->map);
      if (dmap_init(&d->map, 16)) return ORACLE_ERR_NOMEM;
      d->map_ready = 1;
    }
    free(d->tree);
    d->tree = (digest_t*)calloc(d->num_nodes, sizeof(digest_t));
    if (!d->tree) return ORACLE_ERR_NOMEM;
    d->tree_nodes = d->num_nodes;
  }
  if (d->tree_nodes < d->num_nodes) {   /* Kokkos::resize keeps contents, zero-fills the rest */
    digest_t* t = (digest_t*)realloc(d->tree, (uint64_t)d->num_nodes * sizeof(digest_t));
    if (!t) return ORACLE_ERR_NOMEM;
    memset(t + d->tree_nodes, 0, (d->num_nodes - d->tree_nodes) * sizeof(digest_t));
    d->tree = t; d->tree_nodes = d->num_nodes;
  } else if (d->tree_nodes != d->num_nodes) {
    return ORACLE_ERR_ARG;   /* a shrinking buffer makes the reference read past the input */
  }
  /* the reference reserves size + num_nodes (src/tree_approach.cpp:1622-1623); a baseline also
     reserves for the next checkpoint's rule (its own <= num_nodes entries plus num_nodes), so the
     first incremental checkpoint after it does not rehash every entry.  The capacity of this exact
     map changes no output. */
  uint64_t want = d->map.size + d->num_nodes;
  if (baseline && want < 2ull * d->num_nodes) want = 2ull * d->num_nodes;
  if (dmap_rehash(&d->map, want)) return ORACLE_ERR_NOMEM;
  d->first_vec.n = 0; d->shift_vec.n = 0;
  if (baseline) d->baseline_id = d->current_id;
  int rc = dedup(d, data, len, baseline);
  if (rc < 0) return rc;
  int rc2 = collect_diff(d, data, len, diff, diff_len);
  if (rc2 < 0) return rc2;
  d->current_id += 1;
  return rc ? rc : rc2;
}

void oracle_free(void* p) { free(p); }

/* ------------------------------------------------------------------------------------ */
/* Host-view restart: src/tree_approach.cpp:712-1128                                     */
/* ------------------------------------------------------------------------------------ */
typedef struct { uint64_t* k; uint64_t* v; uint8_t* used; uint64_t cap; } u64map_t;
static int u64map_init(u64map_t* m, uint64_t want) {
  m->cap = 2 * want + 16;
  m->k = (uint64_t*)malloc(m->cap * 8); m->v = (uint64_t*)malloc(m->cap * 8);
  m->used = (uint8_t*)calloc(m->cap, 1);
  return (m->k && m->v && m->used) ? ORACLE_OK : ORACLE_ERR_NOMEM;
}
static void u64map_free(u64map_t* m) { free(m->k); free(m->v); free(m->used); }
static void u64map_clear(u64map_t* m) { memset(m->used, 0, m->cap); }
static uint64_t u64h(uint64_t x) { x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; return x; }
static void u64map_insert(u64map_t* m, uint64_t k, uint64_t v) {   /* insert-if-absent */
  uint64_t s = u64h(k) % m->cap;
  while (m->used[s]) { if (m->k[s] == k) return; if (++s == m->cap) s = 0; }
  m->used[s] = 1; m->k[s] = k; m->v[s] = v;
}
static int u64map_get(const u64map_t* m, uint64_t k, uint64_t* v) {
  uint64_t s = u64h(k) % m->cap;
  while (m->used[s]) { if (m->k[s] == k) { *v = m->v[s]; return 1; } if (++s == m->cap) s = 0; }
  return 0;
}
static uint64_t nid_key(uint32_t node, uint32_t tree) { return ((uint64_t)tree << 32) | node; }

typedef struct {
  uint32_t ref_id, chkpt_id; uint64_t datalen; uint32_t chunk_size, num_first, num_prior, num_shift;
  uint64_t first_off, count_off, shift_off, data_off;
} hdr_t;
static int parse_hdr(const uint8_t* b, uint64_t size, hdr_t* h) {
  if (size < 32) return ORACLE_ERR_FORMAT;
  memcpy(&h->ref_id, b, 4); memcpy(&h->chkpt_id, b + 4, 4); memcpy(&h->datalen, b + 8, 8);
  memcpy(&h->chunk_size, b + 16, 4); memcpy(&h->num_first, b + 20, 4);
  memcpy(&h->num_prior, b + 24, 4); memcpy(&h->num_shift, b + 28, 4);
  h->first_off = 32;
  h->count_off = h->first_off + (uint64_t)h->num_first * 4;
  h->shift_off = h->count_off + (uint64_t)h->num_prior * 8;
  h->data_off = h->shift_off + (uint64_t)h->num_shift * 8;
  if (h->data_off > size || h->chunk_size == 0 || h->datalen == 0) return ORACLE_ERR_FORMAT;
  return ORACLE_OK;
}
static uint32_t rd32(const uint8_t* p) { uint32_t v; memcpy(&v, p, 4); return v; }

/* copy with the bounds the reference leaves unchecked */
static int safe_copy(uint8_t* dst, uint64_t dst_len, uint64_t dst_off, const uint8_t* src,
                     uint64_t src_len, uint64_t src_off, uint64_t n) {
  if (dst_off > dst_len || n > dst_len - dst_off || src_off > src_len || n > src_len - src_off)
    return ORACLE_WARN_OOB;
  memcpy(dst + dst_off, src + src_off, n);
  return ORACLE_OK;
}

/* tree id of shift entry i from the (ckpt,count) table: inclusive scan over ids, smallest
 * id whose running count exceeds i (:872-890 main, :1024-1044 older) */
static uint32_t shift_tree(const uint64_t* cum, uint32_t nids, uint64_t i) {
  uint32_t tree = 0;
  for (uint32_t j = nids - 1; j < nids; j--) if (i < cum[j]) tree = j;
  return tree;
}

int oracle_restart(const uint8_t* const* diffs, const uint64_t* sizes, uint32_t count,
                   uint32_t chkpt_idx, uint8_t* out, uint64_t out_len) {
  if (!diffs || !sizes || chkpt_idx >= count || !out) return ORACLE_ERR_ARG;
  hdr_t h;
  const uint8_t* b = diffs[chkpt_idx];
  uint64_t size = sizes[chkpt_idx];
  if (parse_hdr(b, size, &h)) return ORACLE_ERR_FORMAT;
  if (out_len != h.datalen) return ORACLE_ERR_ARG;
  uint64_t nc = h.datalen / h.chunk_size;
  if (nc * h.chunk_size < h.datalen) nc += 1;
  const uint32_t n = (uint32_t)nc, N = 2 * n - 1;
  int warn = ORACLE_OK;
  nodeid_t* node_list = (nodeid_t*)malloc((uint64_t)n * sizeof(nodeid_t));
  uint32_t* chunk_len = (uint32_t*)malloc(((uint64_t)h.num_first + 1) * 4);
  u64map_t dmap, rmap;
  if (!node_list || !chunk_len || u64map_init(&dmap, 2ull * N + 2) || u64map_init(&rmap, 2ull * N + 2)) {
    free(node_list); free(chunk_len); return ORACLE_ERR_NOMEM;
  }
  for (uint32_t i = 0; i < n; i++) node_list[i] = (nodeid_t){UINT32_MAX, UINT32_MAX};
  uint32_t ref_id = h.ref_id, cur_id = h.chkpt_id;
  uint64_t datalen = h.datalen, cs = h.chunk_size;
  const uint8_t* data = b + h.data_off;
  uint64_t data_len = size - h.data_off;
  /* Calculate num chunks + Calc offsets (:797-812) */
  uint32_t run = 0;
  for (uint32_t i = 0; i < h.num_first; i++) {
    uint32_t node = rd32(b + h.first_off + 4 * (uint64_t)i);
    uint32_t len = oracle_num_leaf_descendents(node, N);
    chunk_len[i] = run; run += len;
  }
  /* Restart distinct entries (:822-865) */
  for (uint32_t i = 0; i < h.num_first; i++) {
    uint32_t node = rd32(b + h.first_off + 4 * (uint64_t)i);
    u64map_insert(&dmap, nid_key(node, cur_id), (uint64_t)chunk_len[i] * cs);
    uint32_t start, endl; leaf_range(node, N, &start, &endl);
    uint32_t len = endl - start + 1;
    uint32_t left = 2 * node + 1, right = 2 * node + 2;
    while (left < N) {
      if (right >= N) right = N;
      for (uint32_t j = 0; j <= right - left; j++) {
        uint32_t u = left + j;
        uint32_t leaf = oracle_leftmost_leaf(u, N);
        u64map_insert(&dmap, nid_key(u, cur_id), (uint64_t)(uint32_t)(chunk_len[i] + leaf - start) * cs);
      }
      left = 2 * left + 1; right = 2 * right + 2;
    }
    for (uint32_t j = 0; j < len; j++) {
      uint64_t c = (uint64_t)start - (n - 1) + j;
      if (c < n) node_list[c] = (nodeid_t){(uint32_t)c, cur_id}; else warn = ORACLE_WARN_OOB;
    }
    uint64_t src_offset = (uint64_t)chunk_len[i] * cs;
    uint64_t dst_offset = (uint64_t)(start - (n - 1)) * cs;
    uint64_t datasize = (uint64_t)len * cs;
    if (endl == N - 1) datasize = datalen - dst_offset;
    if (safe_copy(out, out_len, dst_offset, data, data_len, src_offset, datasize)) warn = ORACLE_WARN_OOB;
  }
  /* Load repeat map + Repeat offsets (:871-885) */
  uint64_t* cum = (uint64_t*)calloc((uint64_t)cur_id + 1, 8);
  if (!cum) { warn = ORACLE_ERR_NOMEM; goto fin; }
  for (uint32_t i = 0; i < h.num_prior; i++) {
    uint32_t ck = rd32(b + h.count_off + 8 * (uint64_t)i), cnt = rd32(b + h.count_off + 8 * (uint64_t)i + 4);
    if (ck <= cur_id) cum[ck] = cnt; else warn = ORACLE_WARN_OOB;
  }
  for (uint32_t t = 1; t <= cur_id; t++) cum[t] += cum[t - 1];
  /* Restart shifted duplicates of the main checkpoint (:888-927) */
  for (uint32_t i = 0; i < h.num_shift; i++) {
    uint32_t node = rd32(b + h.shift_off + 8 * (uint64_t)i), prev = rd32(b + h.shift_off + 8 * (uint64_t)i + 4);
    uint32_t tree = shift_tree(cum, cur_id + 1, i);
    uint64_t offset = 0, v;
    if (u64map_get(&dmap, nid_key(prev, tree), &v)) offset = v;
    uint32_t node_start = oracle_leftmost_leaf(node, N);
    uint32_t prev_start = oracle_leftmost_leaf(prev, N);
    uint32_t len = oracle_num_leaf_descendents(prev, N);
    for (uint32_t j = 0; j < len; j++) {
      uint64_t c = (uint64_t)node_start + j - (n - 1);
      if (c < n) node_list[c] = (nodeid_t){prev_start + j, tree}; else warn = ORACLE_WARN_OOB;
    }
    if (tree == cur_id) {
      uint64_t dst_offset = cs * (uint64_t)(node_start - (n - 1));
      uint64_t datasize = cs * (uint64_t)len;
      if ((uint64_t)node_start + len - 1 == N - 1) datasize = out_len - dst_offset;
      if (safe_copy(out, out_len, dst_offset, data, data_len, offset, datasize)) warn = ORACLE_WARN_OOB;
    }
  }
  free(cum); cum = NULL;
  /* Fill same entries (:933-939) */
  for (uint32_t i = 0; i < n; i++)
    if (node_list[i].node == UINT32_MAX) node_list[i] = (nodeid_t){i + n - 1, cur_id - 1};
  /* Older checkpoints (:943-1121) */
  for (int idx = (int)chkpt_idx - 1; idx >= (int)ref_id && idx >= 0; idx--) {
    hdr_t hh;
    const uint8_t* bb = diffs[idx];
    uint64_t bsize = sizes[idx];
    if (parse_hdr(bb, bsize, &hh)) { warn = ORACLE_ERR_FORMAT; goto fin; }
    datalen = hh.datalen; cs = hh.chunk_size;
    ref_id = hh.ref_id; cur_id = hh.chkpt_id;
    const uint8_t* dd = bb + hh.data_off;
    uint64_t dd_len = bsize - hh.data_off;
    u64map_clear(&dmap); u64map_clear(&rmap);
    uint32_t* clen = (uint32_t*)malloc(((uint64_t)hh.num_first + 1) * 4);
    uint64_t* cm = (uint64_t*)calloc((uint64_t)cur_id + 1, 8);
    if (!clen || !cm) { free(clen); free(cm); warn = ORACLE_ERR_NOMEM; goto fin; }
    run = 0;
    for (uint32_t i = 0; i < hh.num_first; i++) {
      uint32_t node = rd32(bb + hh.first_off + 4 * (uint64_t)i);
      uint32_t len = oracle_num_leaf_descendents(node, N);
      clen[i] = run; run += len;
    }
    for (uint32_t i = 0; i < hh.num_first; i++) {          /* :1005-1030 */
      uint32_t node = rd32(bb + hh.first_off + 4 * (uint64_t)i);
      uint64_t offset = (uint64_t)clen[i] * cs;
      u64map_insert(&dmap, nid_key(node, cur_id), offset);
      uint32_t start = oracle_leftmost_leaf(node, N);
      uint32_t left = 2 * node + 1, right = 2 * node + 2;
      while (left < N) {
        if (right >= N) right = N;
        for (uint32_t j = 0; j <= right - left; j++) {
          uint32_t u = left + j;
          uint32_t leaf = oracle_leftmost_leaf(u, N);
          uint64_t leaf_offset = (uint64_t)(uint32_t)(leaf - start) * cs;
          u64map_insert(&dmap, nid_key(u, cur_id), offset + leaf_offset);
        }
        left = 2 * left + 1; right = 2 * right + 2;
      }
    }
    for (uint32_t i = 0; i < hh.num_prior; i++) {            /* :1032-1043 */
      uint32_t ck = rd32(bb + hh.count_off + 8 * (uint64_t)i), cnt = rd32(bb + hh.count_off + 8 * (uint64_t)i + 4);
      if (ck <= cur_id) cm[ck] = cnt; else warn = ORACLE_WARN_OOB;
    }
    for (uint32_t t = 1; t <= cur_id; t++) cm[t] += cm[t - 1];
    for (uint32_t i = 0; i < hh.num_shift; i++) {           /* :1049-1075 */
      uint32_t node = rd32(bb + hh.shift_off + 8 * (uint64_t)i), prev = rd32(bb + hh.shift_off + 8 * (uint64_t)i + 4);
      uint32_t tree = shift_tree(cm, cur_id + 1, i);
      u64map_insert(&rmap, node, nid_key(prev, tree));
      uint32_t curr_start = oracle_leftmost_leaf(node, N);
      uint32_t prev_start = oracle_leftmost_leaf(prev, N);
      uint32_t len = oracle_num_leaf_descendents(node, N);
      for (uint32_t u = 0; u < len; u++) u64map_insert(&rmap, curr_start + u, nid_key(prev_start + u, tree));
    }
    for (uint32_t i = 0; i < n; i++) {                       /* Fill data middle chkpts :1083-1118 */
      if (node_list[i].tree != cur_id) continue;
      nodeid_t id = node_list[i];
      uint64_t v;
      uint64_t dst_offset = (uint64_t)i * cs;
      uint64_t writesize = cs;
      if (dst_offset + writesize > datalen) writesize = datalen - dst_offset;
      if (u64map_get(&dmap, nid_key(id.node, id.tree), &v)) {
        if (safe_copy(out, out_len, dst_offset, dd, dd_len, v, writesize)) warn = ORACLE_WARN_OOB;
      } else if (u64map_get(&rmap, id.node, &v)) {
        nodeid_t prev = {(uint32_t)v, (uint32_t)(v >> 32)};
        if (prev.tree == cur_id) {
          uint64_t src;
          if (u64map_get(&dmap, nid_key(prev.node, prev.tree), &src)) {
            if (safe_copy(out, out_len, dst_offset, dd, dd_len, src, writesize)) warn = ORACLE_WARN_OOB;
          } else {
            warn = ORACLE_WARN_OOB;   /* the reference reads value_at() of a missing key */
          }
        } else {
          node_list[i] = prev;
        }
      } else {
        node_list[i] = (nodeid_t){id.node, cur_id - 1};
      }
    }
    free(clen); free(cm);
  }
fin:
  free(cum);
  free(node_list); free(chunk_len); u64map_free(&dmap); u64map_free(&rmap);
  return warn;
}
