// Restart: rebuild checkpoint `id` from the diffs ref_id..id (host-view restart of the
// reference, src/tree_approach.cpp:712-1128).
//
// The reference keeps two hash maps per diff (NodeID -> data offset for every node under a
// first-occurrence region, node -> source NodeID for every shifted leaf).  Every lookup the
// restart makes is for a leaf, so here both become dense per-chunk arrays:
//   node_list[c] : NodeID the chunk still has to come from (the reference's node_list)
//   dist[c]      : chunk offset of leaf c inside this diff's data section (or absent)
//   rep[c]       : source NodeID of shifted leaf c in this diff (or absent)
// Each diff is processed newest to oldest like the reference; the region lists are expanded
// one thread per chunk after an exclusive scan of the region sizes, and chunk copies use
// 16-byte vectors when both sides are aligned.  Every index and copy is bounds-checked: a
// diff that would make the reference read or write outside a buffer sets DERR_RESTART_RANGE
// and the access is skipped.
#include "restart.cuh"
#include "scan.cuh"

namespace b2d {

constexpr uint32_t R_THREADS = 256;

__device__ __forceinline__ uint32_t rd_u32(const uint8_t* p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}

__device__ __forceinline__ void copy_bytes(uint8_t* dst, const uint8_t* src, uint64_t nb) {
  if ((((uintptr_t)dst | (uintptr_t)src) & 15u) == 0) {
    const uint64_t nv = nb / 16u;
    uint4* d4 = reinterpret_cast<uint4*>(dst);
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
    for (uint64_t i = 0; i < nv; i++) d4[i] = s4[i];
    for (uint64_t i = nv * 16u; i < nb; i++) dst[i] = src[i];
  } else {
    for (uint64_t i = 0; i < nb; i++) dst[i] = src[i];
  }
}

// bounds-checked copy of `nb` bytes: out[dst_off..] <- data section[src_off..]
__device__ __forceinline__ void checked_copy(const RestartArgs& a, uint64_t dst_off, uint64_t src_off, uint64_t nb) {
  const uint64_t data_len = a.diff_size - a.data_off;
  if (dst_off > a.out_len || nb > a.out_len - dst_off || src_off > data_len || nb > data_len - src_off) {
    set_error(a.st, DERR_RESTART_RANGE, 1);
    return;
  }
  copy_bytes(a.out + dst_off, a.diff + a.data_off + src_off, nb);
}

__device__ __forceinline__ uint32_t entry_len(const RestartArgs& a, uint64_t i, int which) {
  if (which == 0) return num_leaf_descendents(rd_u32(a.diff + a.first_off + 4 * i), a.N);
  const uint32_t node = rd_u32(a.diff + a.shift_off + 8 * i);
  const uint32_t prev = rd_u32(a.diff + a.shift_off + 8 * i + 4);
  // the main diff copies num_leaf_descendents(prev) leaves (:906), older diffs map
  // num_leaf_descendents(node) leaves (:1067)
  return num_leaf_descendents(a.is_main ? prev : node, a.N);
}

__global__ void __launch_bounds__(R_THREADS) r_count_kernel(RestartArgs a, int which) {
  __shared__ uint32_t sh[R_THREADS / 32 + 1];
  uint64_t beg, end;
  cta_range(which == 0 ? a.F : a.S, blockIdx.x, gridDim.x, beg, end);
  uint32_t c = 0;
  for (uint64_t i = beg + threadIdx.x; i < end; i += blockDim.x) c += entry_len(a, i, which);
  const uint32_t t = block_reduce_sum(c, sh);
  if (threadIdx.x == 0) a.partial[blockIdx.x] = t;
}

__global__ void __launch_bounds__(1024) r_scan_kernel(RestartArgs a, uint32_t g) {
  __shared__ uint32_t sh[33];
  uint32_t tot;
  const uint32_t i = threadIdx.x;
  const uint32_t v = i < g ? a.partial[i] : 0u;
  const uint32_t e = block_excl_scan(v, sh, &tot);
  if (i < g) a.partial[i] = e;
  if (i == 0) *a.total = tot;
}

__global__ void __launch_bounds__(R_THREADS) r_write_kernel(RestartArgs a, int which) {
  __shared__ uint32_t sh[R_THREADS / 32 + 1];
  uint64_t beg, end;
  cta_range(which == 0 ? a.F : a.S, blockIdx.x, gridDim.x, beg, end);
  uint32_t base = a.partial[blockIdx.x];
  for (uint64_t t0 = beg; t0 < end; t0 += blockDim.x) {
    const uint64_t i = t0 + threadIdx.x;
    const uint32_t len = i < end ? entry_len(a, i, which) : 0u;
    uint32_t tot;
    const uint32_t e = block_excl_scan(len, sh, &tot);
    if (i < end) a.offs[i] = base + e;
    base += tot;
  }
}

__device__ __forceinline__ uint32_t find_entry(const uint32_t* off, uint32_t cnt, uint64_t k) {
  uint32_t lo = 0, hi = cnt;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= k) lo = mid; else hi = mid;
  }
  return lo;
}

// first-occurrence regions: dist[] for every leaf; the main diff also fills node_list and
// copies the chunk (:822-865 main, :1005-1030 older)
__global__ void __launch_bounds__(R_THREADS) r_expand_first_kernel(RestartArgs a) {
  const uint64_t T = *a.total;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < T; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = find_entry(a.offs, a.F, k);
    const uint32_t node = rd_u32(a.diff + a.first_off + 4ull * i);
    const uint32_t start = leftmost_leaf(node, a.N);
    const uint32_t j = (uint32_t)(k - a.offs[i]);
    const uint64_t c = (uint64_t)start - (a.n - 1u) + j;
    if (start < a.n - 1u || c >= a.n) { set_error(a.st, DERR_RESTART_RANGE, 2); continue; }
    const uint32_t off = a.offs[i] + j;   // u32 like the reference (:846, :1018)
    a.dist[c] = off;
    if (a.is_main) {
      a.node_list[c] = make_uint2((uint32_t)c, a.cur_id);
      const uint64_t dst = c * a.cs;
      const uint64_t nb = (c == a.n - 1u) ? a.datalen - dst : a.cs;
      checked_copy(a, dst, (uint64_t)off * a.cs, nb);
    }
  }
}

// Leaves on the shallower level under a region root that spans two depths (only possible
// when the chunk count is not a power of two): the reference inserts them with an offset
// computed in wrapping u32 arithmetic (:844-846, :1016-1018).  Reproduced so later lookups
// of those leaves behave the same.
StraddleQuery straddle_query(uint32_t n) {
  StraddleQuery q;
  q.count = 0;
  if (n < 3 || (n & (n - 1)) == 0) return q;
  uint32_t x = n - 2, y = n - 1;
  while (x != y) {
    if (x > y) x = (x - 1) / 2;
    else y = (y - 1) / 2;
  }
  for (;;) {
    q.anc[q.count++] = x;
    if (x == 0 || q.count == 32) break;
    x = (x - 1) / 2;
  }
  return q;
}

__global__ void r_straddle_find_kernel(RestartArgs a, StraddleQuery q, StraddleInfo* sd) {
  const uint32_t D = node_level(a.N - 1u);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.F; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t node = rd_u32(a.diff + a.first_off + 4 * i);
    bool hit = false;
    for (uint32_t k = 0; k < q.count; k++) hit |= q.anc[k] == node;
    if (!hit) continue;
    // leaves of level D-1 under this root
    const uint32_t k = (D - 1u) - node_level(node);
    const uint64_t lo_all = ((uint64_t)node << k) + (1ull << k) - 1ull;
    const uint64_t hi_all = lo_all + (1ull << k) - 1ull;
    const uint64_t lo = lo_all > (uint64_t)a.n - 1u ? lo_all : (uint64_t)a.n - 1u;
    const uint64_t lvl_end = (1ull << D) - 2ull;
    const uint64_t hi = hi_all < lvl_end ? hi_all : lvl_end;
    if (lo <= hi) {
      sd->root = node;
      sd->region_off = a.offs[i];
      sd->lo = (uint32_t)lo;
      sd->hi = (uint32_t)hi;
      __threadfence();
      sd->present = 1;
    }
  }
}

__global__ void r_straddle_kernel(RestartArgs a, const StraddleInfo* sd) {
  if (!sd->present) return;
  const uint32_t root = sd->root, region_off = sd->region_off, lo = sd->lo, hi = sd->hi;
  const uint32_t start = leftmost_leaf(root, a.N);
  for (uint64_t u = lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u <= hi; u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = u - (a.n - 1u);
    if (c < a.n) a.dist[c] = (uint32_t)(region_off + (uint32_t)u - start);   // zero-extended
  }
}

__device__ __forceinline__ uint32_t shift_tree(const RestartArgs& a, uint64_t i) {
  // smallest checkpoint id whose inclusive running count exceeds i, else 0 (:879-885)
  uint32_t lo = 0, hi = a.ncum;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a.cum[mid] > i) hi = mid; else lo = mid + 1;
  }
  return lo < a.ncum ? lo : 0u;
}

// shifted-duplicate entries (:888-927 main, :1049-1075 older)
__global__ void __launch_bounds__(R_THREADS) r_expand_shift_kernel(RestartArgs a) {
  const uint64_t T = *a.total;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < T; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = find_entry(a.offs, a.S, k);
    const uint32_t node = rd_u32(a.diff + a.shift_off + 8ull * i);
    const uint32_t prev = rd_u32(a.diff + a.shift_off + 8ull * i + 4);
    const uint32_t j = (uint32_t)(k - a.offs[i]);
    const uint32_t tree = shift_tree(a, i);
    const uint32_t node_start = leftmost_leaf(node, a.N);
    const uint32_t prev_start = leftmost_leaf(prev, a.N);
    const uint64_t c = (uint64_t)node_start + j - (a.n - 1u);
    if (node_start < a.n - 1u || c >= a.n) { set_error(a.st, DERR_RESTART_RANGE, 3); continue; }
    if (a.is_main) {
      a.node_list[c] = make_uint2(prev_start + j, tree);
      if (tree == a.cur_id) {
        // offset of NodeID(prev, cur) = offset of prev's leftmost leaf; absent -> 0 (:898-901)
        uint64_t base = 0;
        const uint64_t pc = (uint64_t)prev_start - (a.n - 1u);
        if (prev_start >= a.n - 1u && pc < a.n && a.dist[pc] != R_ABSENT) base = (uint64_t)a.dist[pc] * a.cs;
        const uint64_t dst = c * a.cs;
        const uint64_t nb = (c == a.n - 1u) ? a.out_len - dst : a.cs;
        checked_copy(a, dst, base + (uint64_t)j * a.cs, nb);
      }
    } else {
      a.rep[c] = make_uint2(prev_start + j, tree);
    }
  }
}

// chunks named by no region of the main diff come from the previous checkpoint (:933-939)
__global__ void r_fill_same_kernel(RestartArgs a) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < a.n; c += (uint64_t)gridDim.x * blockDim.x) {
    if (a.node_list[c].x == 0xffffffffu) a.node_list[c] = make_uint2((uint32_t)c + a.n - 1u, a.cur_id - 1u);
  }
}

// resolve chunks still owed by an older diff (:1083-1118)
__global__ void r_fill_older_kernel(RestartArgs a) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < a.n; c += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 id = a.node_list[c];
    if (id.y != a.cur_id) continue;
    const uint64_t dst = c * a.cs;
    uint64_t ws = a.cs;
    if (dst + ws > a.datalen) ws = a.datalen - dst;
    const uint64_t lc = (uint64_t)id.x - (a.n - 1u);
    const bool leaf = id.x >= a.n - 1u && lc < a.n;
    if (leaf && a.dist[lc] != R_ABSENT) {
      checked_copy(a, dst, (uint64_t)a.dist[lc] * a.cs, ws);
    } else if (leaf && a.rep[lc].x != 0xffffffffu) {
      const uint2 prev = a.rep[lc];
      if (prev.y == a.cur_id) {
        const uint64_t pc = (uint64_t)prev.x - (a.n - 1u);
        if (prev.x >= a.n - 1u && pc < a.n && a.dist[pc] != R_ABSENT) checked_copy(a, dst, (uint64_t)a.dist[pc] * a.cs, ws);
        else set_error(a.st, DERR_RESTART_RANGE, 4);
      } else {
        a.node_list[c] = prev;
      }
    } else {
      a.node_list[c] = make_uint2(id.x, a.cur_id - 1u);
    }
  }
}

// running shift counts per checkpoint id from a device-resident diff's (ckpt, count) table:
// the last row for an id wins, then an inclusive scan over ids (:871-885); rows naming an id
// beyond the diff's own are outside the reference's array and are reported
__global__ void r_cum_kernel(RestartArgs a) {
  unsigned long long* cum = const_cast<unsigned long long*>(a.cum);
  for (uint32_t t = threadIdx.x; t < a.ncum; t += blockDim.x) cum[t] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < a.P; i++) {
      const uint32_t ck = rd_u32(a.diff + a.count_off + 8ull * i);
      const uint32_t cnt = rd_u32(a.diff + a.count_off + 8ull * i + 4);
      if (ck < a.ncum) cum[ck] = cnt;
      else set_error(a.st, DERR_RESTART_RANGE, 5);
    }
    unsigned long long run = 0;
    for (uint32_t t = 0; t < a.ncum; t++) {
      run += cum[t];
      cum[t] = run;
    }
  }
}

cudaError_t launch_restart_cum(const RestartArgs& a, cudaStream_t s) {
  r_cum_kernel<<<1, 256, 0, s>>>(a);
  return cudaGetLastError();
}

static uint32_t grid_for(uint64_t work, int sm_count) {
  uint64_t b = ceil_div_u64(work ? work : 1, R_THREADS);
  const uint64_t cap = (uint64_t)sm_count * 8u;
  return (uint32_t)(b > cap ? cap : b);
}

cudaError_t launch_restart_init(const RestartArgs& a, int sm_count, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(a.node_list, 0xff, sizeof(uint2) * (size_t)a.n, s);
  (void)sm_count;
  return e;
}

cudaError_t launch_restart_diff(const RestartArgs& a, StraddleInfo* sd, int sm_count, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(a.dist, 0xff, sizeof(unsigned long long) * (size_t)a.n, s);
  if (e != cudaSuccess) return e;
  if (!a.is_main) {
    e = cudaMemsetAsync(a.rep, 0xff, sizeof(uint2) * (size_t)a.n, s);
    if (e != cudaSuccess) return e;
  }
  const uint32_t g = SCAN_GRID;
  // first-occurrence regions
  r_count_kernel<<<g, R_THREADS, 0, s>>>(a, 0);
  r_scan_kernel<<<1, 1024, 0, s>>>(a, g);
  r_write_kernel<<<g, R_THREADS, 0, s>>>(a, 0);
  r_expand_first_kernel<<<grid_for(a.n, sm_count), R_THREADS, 0, s>>>(a);
  const StraddleQuery q = straddle_query(a.n);
  if (q.count) {
    e = cudaMemsetAsync(sd, 0, sizeof(StraddleInfo), s);
    if (e != cudaSuccess) return e;
    r_straddle_find_kernel<<<grid_for(a.F, sm_count), R_THREADS, 0, s>>>(a, q, sd);
    r_straddle_kernel<<<(uint32_t)sm_count * 4u, R_THREADS, 0, s>>>(a, sd);
  }
  // shifted duplicates
  r_count_kernel<<<g, R_THREADS, 0, s>>>(a, 1);
  r_scan_kernel<<<1, 1024, 0, s>>>(a, g);
  r_write_kernel<<<g, R_THREADS, 0, s>>>(a, 1);
  r_expand_shift_kernel<<<grid_for(a.n, sm_count), R_THREADS, 0, s>>>(a);
  if (a.is_main) r_fill_same_kernel<<<grid_for(a.n, sm_count), R_THREADS, 0, s>>>(a);
  else r_fill_older_kernel<<<grid_for(a.n, sm_count), R_THREADS, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace b2d
