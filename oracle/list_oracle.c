/*
 * list_oracle.c -- CPU restatement of the reference ListDeduplicator (list approach) used
 * ONLY as the correctness checker.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * / reference arm may load this library.  The product (libb200dedup.so) never links,
 * loads or calls it, and has no CPU fallback.
 *
 * Every function follows the reference source as if the Kokkos dispatches ran sequentially
 * (one thread, ascending index), which is the canonical output order the GPU library must
 * reproduce:
 *   per-chunk dedup ... src/list_approach.cpp:23-77 (digest differs from the chunk's previous
 *                       digest -> insert; success = first occurrence, existing = shifted
 *                       duplicate; the chunk's list entry takes the new digest)
 *   diff assembly ..... src/list_approach.cpp:79-257 (first list in push order, repeat table
 *                       ascending by checkpoint, shifted pairs stably sorted by the source
 *                       checkpoint, data of the first occurrences in list order)
 *   checkpoint ........ src/list_approach.cpp:843-931 (a baseline resets the digest list to
 *                       zeros and empties the map) plus the current_id += 1 of :954-962
 *   host-view restart . src/list_approach.cpp:259-586
 * The chunk digests of a checkpoint are computed up front (optionally with OpenMP threads);
 * hashing is a pure function of the chunk bytes, so this changes no result.
 *
 * Memory safety: where the reference would index outside a buffer (corrupt diffs), the oracle
 * skips the access and reports ORACLE_WARN_OOB.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_OK 0
#define ORACLE_ERR_ARG (-1)
#define ORACLE_ERR_NOMEM (-2)
#define ORACLE_ERR_FORMAT (-3)
#define ORACLE_WARN_OOB 2

void oracle_hash(int kind, const uint8_t* data, uint64_t len, uint8_t out[16]);   /* tree_oracle.c */

typedef struct { uint8_t b[16]; } ldigest_t;
typedef struct { uint32_t node, tree; } lnodeid_t;   /* include/map_helpers.hpp:38-58 */

/* digest -> NodeID, insert-if-absent (the DigestNodeIDDeviceMap contract) */
typedef struct {
  ldigest_t* keys;
  lnodeid_t* vals;
  uint8_t* used;
  uint64_t cap, size;
} lmap_t;

static uint64_t lmap_slot(const ldigest_t* k, uint64_t cap) {
  uint64_t a, b;
  memcpy(&a, k->b, 8);
  memcpy(&b, k->b + 8, 8);
  uint64_t h = a ^ (b * 0x9E3779B97F4A7C15ULL);
  h ^= h >> 31;
  return h % cap;
}
static int lmap_init(lmap_t* m, uint64_t cap) {
  memset(m, 0, sizeof *m);
  if (cap < 16) cap = 16;
  m->keys = (ldigest_t*)malloc(cap * sizeof(ldigest_t));
  m->vals = (lnodeid_t*)malloc(cap * sizeof(lnodeid_t));
  m->used = (uint8_t*)calloc(cap, 1);
  if (!m->keys || !m->vals || !m->used) return ORACLE_ERR_NOMEM;
  m->cap = cap;
  return ORACLE_OK;
}
static void lmap_free(lmap_t* m) {
  free(m->keys);
  free(m->vals);
  free(m->used);
  memset(m, 0, sizeof *m);
}
static int64_t lmap_find(const lmap_t* m, const ldigest_t* k) {
  if (!m->cap) return -1;
  uint64_t s = lmap_slot(k, m->cap);
  while (m->used[s]) {
    if (memcmp(m->keys[s].b, k->b, 16) == 0) return (int64_t)s;
    if (++s == m->cap) s = 0;
  }
  return -1;
}
static int64_t lmap_insert_raw(lmap_t* m, const ldigest_t* k, lnodeid_t v, int* inserted) {
  uint64_t s = lmap_slot(k, m->cap);
  while (m->used[s]) {
    if (memcmp(m->keys[s].b, k->b, 16) == 0) {
      *inserted = 0;
      return (int64_t)s;
    }
    if (++s == m->cap) s = 0;
  }
  m->used[s] = 1;
  m->keys[s] = *k;
  m->vals[s] = v;
  m->size++;
  *inserted = 1;
  return (int64_t)s;
}
static int lmap_reserve(lmap_t* m, uint64_t want) {   /* capacity is internal: load <= 1/2 */
  if (m->cap && 2 * want + 16 <= m->cap) return ORACLE_OK;
  lmap_t n;
  if (lmap_init(&n, 3 * want + 16)) return ORACLE_ERR_NOMEM;
  for (uint64_t s = 0; s < m->cap; s++)
    if (m->used[s]) {
      int ins;
      lmap_insert_raw(&n, &m->keys[s], m->vals[s], &ins);
    }
  lmap_free(m);
  *m = n;
  return ORACLE_OK;
}

typedef struct {
  uint32_t* v;
  uint64_t n, cap;
} lvec_t;
static int lvec_push(lvec_t* v, uint32_t x) {
  if (v->n == v->cap) {
    uint64_t c = v->cap ? 2 * v->cap : 64;
    uint32_t* p = (uint32_t*)realloc(v->v, c * sizeof(uint32_t));
    if (!p) return ORACLE_ERR_NOMEM;
    v->v = p;
    v->cap = c;
  }
  v->v[v->n++] = x;
  return ORACLE_OK;
}

/* include/list_approach.hpp: chunk size, ids, the per-chunk digest list, the map, the vectors */
typedef struct oracle_list {
  uint32_t chunk_size;
  int hash_kind;
  int threads;
  uint32_t current_id, baseline_id;
  uint64_t data_len;
  uint32_t num_chunks;
  ldigest_t* list;
  uint64_t list_len;
  lmap_t map;
  lvec_t first_vec, shift_vec;
  uint64_t datasizes[2];
} oracle_list;

oracle_list* oracle_list_create(uint32_t chunk_size, int hash_kind) {
  if (chunk_size == 0) return NULL;
  oracle_list* d = (oracle_list*)calloc(1, sizeof(oracle_list));
  if (!d) return NULL;
  d->chunk_size = chunk_size;   /* src/list_approach.cpp:5-9 */
  d->hash_kind = hash_kind;
  d->threads = 1;
  return d;
}
void oracle_list_destroy(oracle_list* d) {
  if (!d) return;
  free(d->list);
  lmap_free(&d->map);
  free(d->first_vec.v);
  free(d->shift_vec.v);
  free(d);
}
void oracle_list_set_threads(oracle_list* d, int t) { d->threads = t < 1 ? 1 : t; }
uint64_t oracle_list_num_first_ocur(const oracle_list* d) { return d->first_vec.n; }
uint64_t oracle_list_num_shift_dupl(const oracle_list* d) { return d->shift_vec.n; }
uint32_t oracle_list_current_id(const oracle_list* d) { return d->current_id; }
void oracle_list_datasizes(const oracle_list* d, uint64_t out[2]) {
  out[0] = d->datasizes[0];
  out[1] = d->datasizes[1];
}

/* src/list_approach.cpp:23-77 */
static int list_dedup(oracle_list* d, const uint8_t* data, uint64_t len) {
  const uint32_t n = d->num_chunks, cur = d->current_id;
  const uint64_t cs = d->chunk_size;
  ldigest_t* dig = (ldigest_t*)malloc((uint64_t)n * sizeof(ldigest_t) + 1);
  if (!dig) return ORACLE_ERR_NOMEM;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(d->threads)
#endif
  for (int64_t c = 0; c < (int64_t)n; c++) {
    const uint64_t off = (uint64_t)c * cs;
    const uint64_t nb = (c == (int64_t)n - 1) ? len - off : cs;
    oracle_hash(d->hash_kind, data + off, nb, dig[c].b);
  }
  int rc = ORACLE_OK;
  for (uint32_t c = 0; c < n; c++) {
    if (memcmp(d->list[c].b, dig[c].b, 16) == 0) continue;   /* digests_same: unchanged */
    int ins;
    lmap_insert_raw(&d->map, &dig[c], (lnodeid_t){c, cur}, &ins);
    rc = ins ? lvec_push(&d->first_vec, c) : lvec_push(&d->shift_vec, c);
    if (rc) break;
    d->list[c] = dig[c];
  }
  free(dig);
  return rc;
}

/* src/list_approach.cpp:79-257 */
static int list_collect_diff(oracle_list* d, const uint8_t* data, uint64_t len, uint8_t** out, uint64_t* out_len) {
  const uint32_t n = d->num_chunks, cur = d->current_id;
  const uint64_t cs = d->chunk_size;
  const uint64_t F = d->first_vec.n, S = d->shift_vec.n;
  uint64_t* prior = (uint64_t*)calloc((uint64_t)cur + 1, sizeof(uint64_t));
  uint32_t* skey = (uint32_t*)malloc((S + 1) * sizeof(uint32_t));
  uint32_t* sprev = (uint32_t*)malloc((S + 1) * sizeof(uint32_t));
  uint8_t* buf = NULL;
  int rc = ORACLE_OK;
  if (!prior || !skey || !sprev) {
    rc = ORACLE_ERR_NOMEM;
    goto done;
  }
  /* Count shifted dupl (:106-114): the map entry of the chunk's (new) digest */
  for (uint64_t i = 0; i < S; i++) {
    const uint32_t c = d->shift_vec.v[i];
    const int64_t s = lmap_find(&d->map, &d->list[c]);
    const lnodeid_t e = s >= 0 ? d->map.vals[s] : (lnodeid_t){0, 0};
    if (e.tree <= cur) prior[e.tree] += 1;
    skey[i] = e.tree;
    sprev[i] = e.node;
  }
  uint32_t num_prior = 0;   /* chkpts_needed.count() */
  for (uint32_t t = 0; t <= cur; t++) num_prior += prior[t] > 0;
  /* sizes and offsets (:125-137) */
  const uint64_t buffer_len = 32 + F * (4 + cs) + (uint64_t)num_prior * 8 + S * 8;
  const uint64_t data_offset = 32 + F * 4 + (uint64_t)num_prior * 8 + S * 8;
  buf = (uint8_t*)calloc(buffer_len, 1);   /* fresh view: zero-filled */
  if (!buf) {
    rc = ORACLE_ERR_NOMEM;
    goto done;
  }
  /* first occurrence metadata (:149-153) */
  for (uint64_t i = 0; i < F; i++) memcpy(buf + 32 + 4 * i, &d->first_vec.v[i], 4);
  /* repeat table (:155-165): one row per checkpoint with entries, ascending */
  uint64_t pos = 32 + 4 * F;
  for (uint32_t t = 0; t <= cur; t++) {
    if (!prior[t]) continue;
    const uint32_t cnt = (uint32_t)prior[t];
    memcpy(buf + pos, &t, 4);
    memcpy(buf + pos + 4, &cnt, 4);
    pos += 8;
  }
  /* shifted pairs (node, source node), stably sorted by source checkpoint (:174-218) */
  uint64_t w = 0;
  const uint64_t shift_offset = 32 + 4 * F + 8ull * num_prior;
  for (uint32_t t = 0; t <= cur; t++) {
    if (!prior[t]) continue;
    for (uint64_t i = 0; i < S; i++) {
      if (skey[i] != t) continue;
      memcpy(buf + shift_offset + 8 * w, &d->shift_vec.v[i], 4);
      memcpy(buf + shift_offset + 8 * w + 4, &sprev[i], 4);
      w++;
    }
  }
  /* data of the first occurrences, short last chunk zero-padded (:221-235) */
  for (uint64_t i = 0; i < F; i++) {
    const uint32_t c = d->first_vec.v[i];
    const uint64_t src = (uint64_t)c * cs;
    const uint64_t wsz = (c == n - 1) ? len - src : cs;
    if (c >= n || src + wsz > len) {
      rc = ORACLE_WARN_OOB;
      continue;
    }
    memcpy(buf + data_offset + i * cs, data + src, wsz);
  }
  /* header (:238-244) */
  {
    uint32_t h32;
    h32 = d->baseline_id;
    memcpy(buf + 0, &h32, 4);
    h32 = cur;
    memcpy(buf + 4, &h32, 4);
    memcpy(buf + 8, &len, 8);
    h32 = d->chunk_size;
    memcpy(buf + 16, &h32, 4);
    h32 = (uint32_t)F;
    memcpy(buf + 20, &h32, 4);
    h32 = num_prior;
    memcpy(buf + 24, &h32, 4);
    h32 = (uint32_t)S;
    memcpy(buf + 28, &h32, 4);
  }
  d->datasizes[0] = cs * F;   /* (:253-256) */
  d->datasizes[1] = buffer_len - cs * F;
  *out = buf;
  *out_len = buffer_len;
  buf = NULL;
done:
  free(prior);
  free(skey);
  free(sprev);
  free(buf);
  return rc;
}

/* src/list_approach.cpp:843-931 and the current_id += 1 of :954-962 */
int oracle_list_checkpoint(oracle_list* d, const uint8_t* data, uint64_t len, int make_baseline, uint8_t** diff,
                           uint64_t* diff_len) {
  if (!d || !diff || !diff_len || len == 0) return ORACLE_ERR_ARG;
  uint64_t nc = len / d->chunk_size;
  if (nc * d->chunk_size < len) nc += 1;
  if (nc > 0x7fffffffULL) return ORACLE_ERR_ARG;
  d->data_len = len;
  d->num_chunks = (uint32_t)nc;
  if (make_baseline) {   /* fresh list (all-zero digests) and an empty map */
    free(d->list);
    d->list = (ldigest_t*)calloc(nc, sizeof(ldigest_t));
    if (!d->list) return ORACLE_ERR_NOMEM;
    d->list_len = nc;
    lmap_free(&d->map);
  }
  d->first_vec.n = 0;
  d->shift_vec.n = 0;
  if (d->list_len < nc) {   /* Kokkos::resize keeps contents, zero-fills the rest */
    ldigest_t* l = (ldigest_t*)realloc(d->list, nc * sizeof(ldigest_t));
    if (!l) return ORACLE_ERR_NOMEM;
    memset(l + d->list_len, 0, (nc - d->list_len) * sizeof(ldigest_t));
    d->list = l;
    d->list_len = nc;
  }
  /* reserve for this checkpoint (size + chunks) and, on a baseline, also for the next one, so the
     first incremental checkpoint does not rehash every entry; capacity changes no output */
  uint64_t want = d->map.size + nc;
  if ((d->current_id == 0 || make_baseline) && want < 2 * nc) want = 2 * nc;
  if (lmap_reserve(&d->map, want)) return ORACLE_ERR_NOMEM;
  if (d->current_id == 0 || make_baseline) d->baseline_id = d->current_id;
  int rc = list_dedup(d, data, len);
  if (rc < 0) return rc;
  rc = list_collect_diff(d, data, len, diff, diff_len);
  if (rc < 0) return rc;
  d->current_id += 1;
  return rc;
}

/* ------------------------------------------------------------------------------------ */
/* Host-view restart: src/list_approach.cpp:259-586                                      */
/* ------------------------------------------------------------------------------------ */
typedef struct {
  uint64_t* k;
  uint64_t* v;
  uint8_t* used;
  uint64_t cap;
} lkv_t;
static int lkv_init(lkv_t* m, uint64_t want) {
  m->cap = 2 * want + 16;
  m->k = (uint64_t*)malloc(m->cap * 8);
  m->v = (uint64_t*)malloc(m->cap * 8);
  m->used = (uint8_t*)calloc(m->cap, 1);
  return (m->k && m->v && m->used) ? ORACLE_OK : ORACLE_ERR_NOMEM;
}
static void lkv_free(lkv_t* m) {
  free(m->k);
  free(m->v);
  free(m->used);
  memset(m, 0, sizeof *m);
}
static uint64_t lkv_h(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  return x;
}
static void lkv_insert(lkv_t* m, uint64_t k, uint64_t v) {   /* insert-if-absent */
  uint64_t s = lkv_h(k) % m->cap;
  while (m->used[s]) {
    if (m->k[s] == k) return;
    if (++s == m->cap) s = 0;
  }
  m->used[s] = 1;
  m->k[s] = k;
  m->v[s] = v;
}
static int lkv_get(const lkv_t* m, uint64_t k, uint64_t* v) {
  uint64_t s = lkv_h(k) % m->cap;
  while (m->used[s]) {
    if (m->k[s] == k) {
      *v = m->v[s];
      return 1;
    }
    if (++s == m->cap) s = 0;
  }
  return 0;
}
static uint64_t lnid(uint32_t node, uint32_t tree) { return ((uint64_t)tree << 32) | node; }
static uint32_t lrd32(const uint8_t* p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}

typedef struct {
  uint32_t ref_id, chkpt_id;
  uint64_t datalen;
  uint32_t chunk_size, num_first, num_prior, num_shift;
  uint64_t first_off, count_off, shift_off, data_off;
} lhdr_t;
static int lparse(const uint8_t* b, uint64_t size, lhdr_t* h) {
  if (size < 32) return ORACLE_ERR_FORMAT;
  memcpy(&h->ref_id, b, 4);
  memcpy(&h->chkpt_id, b + 4, 4);
  memcpy(&h->datalen, b + 8, 8);
  memcpy(&h->chunk_size, b + 16, 4);
  memcpy(&h->num_first, b + 20, 4);
  memcpy(&h->num_prior, b + 24, 4);
  memcpy(&h->num_shift, b + 28, 4);
  h->first_off = 32;   /* (:311-314) */
  h->count_off = h->first_off + (uint64_t)h->num_first * 4;
  h->shift_off = h->count_off + (uint64_t)h->num_prior * 8;
  h->data_off = h->shift_off + (uint64_t)h->num_shift * 8;
  if (h->data_off > size || h->chunk_size == 0 || h->datalen == 0) return ORACLE_ERR_FORMAT;
  return ORACLE_OK;
}
static int lcopy(uint8_t* dst, uint64_t dst_len, uint64_t dst_off, const uint8_t* src, uint64_t src_len,
                 uint64_t src_off, uint64_t nb) {
  if (dst_off > dst_len || nb > dst_len - dst_off || src_off > src_len || nb > src_len - src_off)
    return ORACLE_WARN_OOB;
  memcpy(dst + dst_off, src + src_off, nb);
  return ORACLE_OK;
}
/* running counts per checkpoint id from the (ckpt, count) table; the tree of shift entry i is
 * the smallest id whose running count exceeds i (:344-357, :382-389) */
static int lcum(const uint8_t* b, const lhdr_t* h, uint64_t* cum) {
  int warn = ORACLE_OK;
  for (uint32_t i = 0; i < h->num_prior; i++) {
    const uint32_t ck = lrd32(b + h->count_off + 8ull * i), cnt = lrd32(b + h->count_off + 8ull * i + 4);
    if (ck <= h->chkpt_id) cum[ck] = cnt;
    else warn = ORACLE_WARN_OOB;
  }
  for (uint32_t t = 1; t <= h->chkpt_id; t++) cum[t] += cum[t - 1];
  return warn;
}
static uint32_t ltree(const uint64_t* cum, uint32_t nids, uint64_t i) {
  uint32_t tree = 0;
  for (uint32_t j = nids - 1; j < nids; j--)
    if (i < cum[j]) tree = j;
  return tree;
}

int oracle_list_restart(const uint8_t* const* diffs, const uint64_t* sizes, uint32_t count, uint32_t chkpt_idx,
                        uint8_t* out, uint64_t out_len) {
  if (!diffs || !sizes || chkpt_idx >= count || !out) return ORACLE_ERR_ARG;
  lhdr_t h;
  const uint8_t* b = diffs[chkpt_idx];
  if (lparse(b, sizes[chkpt_idx], &h)) return ORACLE_ERR_FORMAT;
  if (out_len != h.datalen) return ORACLE_ERR_ARG;
  uint64_t nc = h.datalen / h.chunk_size;
  if (nc * h.chunk_size < h.datalen) nc += 1;
  const uint32_t n = (uint32_t)nc;
  int warn = ORACLE_OK;
  lnodeid_t* node_list = (lnodeid_t*)malloc((uint64_t)n * sizeof(lnodeid_t));
  uint64_t* cum = (uint64_t*)calloc((uint64_t)h.chkpt_id + 1, 8);
  lkv_t first = {0}, rep = {0};
  if (!node_list || !cum || lkv_init(&first, (uint64_t)n + 1) || lkv_init(&rep, (uint64_t)n + 1)) {
    warn = ORACLE_ERR_NOMEM;
    goto fin;
  }
  for (uint32_t i = 0; i < n; i++) node_list[i] = (lnodeid_t){UINT32_MAX, UINT32_MAX};   /* NodeID() */
  uint32_t ref_id = h.ref_id, cur_id = h.chkpt_id;
  uint64_t datalen = h.datalen, cs = h.chunk_size;
  const uint8_t* data = b + h.data_off;
  const uint64_t data_len = sizes[chkpt_idx] - h.data_off;
  /* first occurrences of the main diff (:331-351) */
  for (uint32_t i = 0; i < h.num_first; i++) {
    const uint32_t node = lrd32(b + h.first_off + 4ull * i);
    lkv_insert(&first, lnid(node, cur_id), (uint64_t)i * cs);
    if (node >= n) {
      warn = ORACLE_WARN_OOB;
      continue;
    }
    node_list[node] = (lnodeid_t){node, cur_id};
    const uint64_t dst = (uint64_t)node * cs;
    const uint64_t nb = (node == n - 1) ? datalen - dst : cs;
    if (lcopy(out, out_len, dst, data, data_len, (uint64_t)i * cs, nb)) warn = ORACLE_WARN_OOB;
  }
  if (lcum(b, &h, cum)) warn = ORACLE_WARN_OOB;
  /* shifted duplicates of the main diff (:371-408) */
  for (uint32_t i = 0; i < h.num_shift; i++) {
    const uint32_t node = lrd32(b + h.shift_off + 8ull * i), prev = lrd32(b + h.shift_off + 8ull * i + 4);
    const uint32_t tree = ltree(cum, cur_id + 1, i);
    uint64_t src = 0, v;
    if (lkv_get(&first, lnid(prev, tree), &v)) src = v;
    if (node >= n) {
      warn = ORACLE_WARN_OOB;
      continue;
    }
    node_list[node] = (lnodeid_t){prev, tree};
    if (tree == cur_id) {
      const uint64_t dst = (uint64_t)node * cs;
      const uint64_t nb = (node == n - 1) ? datalen - dst : cs;
      if (lcopy(out, out_len, dst, data, data_len, src, nb)) warn = ORACLE_WARN_OOB;
    }
  }
  /* chunks the main diff does not name (:414-422) */
  for (uint32_t i = 0; i < n; i++)
    if (node_list[i].node == UINT32_MAX) node_list[i] = (lnodeid_t){i, cur_id - 1};
  /* older diffs, newest first (:427-578) */
  for (int idx = (int)chkpt_idx - 1; idx >= (int)ref_id && idx < (int)chkpt_idx; idx--) {
    lhdr_t hh;
    const uint8_t* bb = diffs[idx];
    const uint64_t bsize = sizes[idx];
    if (lparse(bb, bsize, &hh)) {
      warn = ORACLE_ERR_FORMAT;
      goto fin;
    }
    const uint32_t current_id = hh.chkpt_id;
    ref_id = hh.ref_id;
    cur_id = hh.chkpt_id;
    datalen = hh.datalen;
    cs = hh.chunk_size;
    const uint8_t* dd = bb + hh.data_off;
    const uint64_t dd_len = bsize - hh.data_off;
    lkv_free(&first);
    lkv_free(&rep);
    uint64_t* cm = (uint64_t*)calloc((uint64_t)cur_id + 1, 8);
    if (!cm || lkv_init(&first, (uint64_t)hh.num_first + 1) || lkv_init(&rep, (uint64_t)hh.num_shift + 1)) {
      free(cm);
      warn = ORACLE_ERR_NOMEM;
      goto fin;
    }
    for (uint32_t i = 0; i < hh.num_first; i++)   /* (:478-482) */
      lkv_insert(&first, lnid(lrd32(bb + hh.first_off + 4ull * i), cur_id), (uint64_t)i * cs);
    if (lcum(bb, &hh, cm)) warn = ORACLE_WARN_OOB;
    for (uint32_t i = 0; i < hh.num_shift; i++) {   /* (:501-513) */
      const uint32_t node = lrd32(bb + hh.shift_off + 8ull * i), prev = lrd32(bb + hh.shift_off + 8ull * i + 4);
      lkv_insert(&rep, node, lnid(prev, ltree(cm, cur_id + 1, i)));
    }
    for (uint32_t i = 0; i < n; i++) {   /* (:516-575) */
      if (node_list[i].tree != current_id) continue;
      const lnodeid_t id = node_list[i];
      const uint64_t dst = (uint64_t)i * cs;
      uint64_t ws = cs;
      if (dst + ws > datalen) ws = datalen - dst;
      uint64_t v;
      if (lkv_get(&first, lnid(id.node, id.tree), &v)) {
        if (lcopy(out, out_len, dst, dd, dd_len, v, ws)) warn = ORACLE_WARN_OOB;
      } else if (lkv_get(&rep, id.node, &v)) {
        const lnodeid_t prev = {(uint32_t)v, (uint32_t)(v >> 32)};
        if (prev.tree == current_id) {
          uint64_t src;
          if (lkv_get(&first, lnid(prev.node, prev.tree), &src)) {
            if (lcopy(out, out_len, dst, dd, dd_len, src, ws)) warn = ORACLE_WARN_OOB;
          } else {
            warn = ORACLE_WARN_OOB;   /* the reference reads value_at() of a missing key */
          }
        } else {
          node_list[i] = prev;
        }
      } else {
        node_list[i] = (lnodeid_t){id.node, current_id - 1};
      }
    }
    free(cm);
  }
fin:
  free(node_list);
  free(cum);
  lkv_free(&first);
  lkv_free(&rep);
  return warn;
}
