// Restart kernel arguments (see restart.cu).
#pragma once
#include "common.cuh"
#include "dedup_kernels.cuh"

namespace b2d {

// One diff's lookups, dense over the leaves of the restarted checkpoint.  An entry means
// something only where its bit in flag[c] is set (the flags are cleared for each diff, the
// arrays are not):
//   dist[c] (flag bit 0) : chunk offset of leaf c inside the diff's data section (u32, like
//                          the reference, which computes some of these offsets in wrapping u32
//                          arithmetic)
//   rep[c]  (flag bit 1) : source NodeID of shifted leaf c
constexpr uint8_t R_HAS_DIST = 1, R_HAS_REP = 2;
struct RestartSlot {
  uint32_t* dist;
  uint2* rep;
  uint8_t* flag;
};

// expansion of one diff's region lists
struct RestartArgs {
  const uint8_t* diff;     // one diff (header at offset 0 of this pointer)
  uint64_t diff_size;
  uint64_t first_off, count_off, shift_off, data_off;   // byte offsets from `diff`
  uint32_t F, P, S;
  uint32_t cur_id;         // chkpt_id of this diff's header
  uint64_t datalen;        // this diff's header datalen
  uint32_t cs;             // this diff's header chunk size
  uint32_t n, N;           // chunks / nodes of the checkpoint being restarted
  int is_main;
  uint8_t* out;            // restart buffer (device)
  uint64_t out_len;        // datalen of the checkpoint being restarted
  uint2* node_list;        // n: NodeID each chunk named by the main diff still comes from
  uint8_t* mflag;          // n: chunk named by the main diff
  RestartSlot slot;        // this diff's lookups
  const unsigned long long* cum;   // inclusive shift counts per checkpoint id (ncum entries)
  uint32_t ncum;
  uint32_t* offs;          // per region entry: exclusive offset of its first chunk
  uint32_t* rstart;        // per region entry: leftmost leaf of the region's node
  uint32_t* pstart;        // per shift entry: leftmost leaf of the source node
  uint32_t* rtree;         // per shift entry: source checkpoint id
  uint32_t* partial;       // SCAN_GRID
  unsigned long long* total;
  DevStatus* st;
  // added to every node id read from the diff: list-approach diffs name chunks, which the
  // restart handles as the leaves n-1+c of the same heap (0 for tree diffs)
  uint32_t id_bias;
  // chunk copies (set by launch_restart_diff): piece width in bytes (16/8/4, dividing the chunk
  // size and the alignment of `out` and of the data section; 0: one lane copies a whole chunk),
  // pieces per chunk and its log2 (0xff when not a power of two)
  uint32_t width, per, per_log2;
};

// Older diffs resolved by one walk over the chunks, newest first.
constexpr uint32_t RESTART_WINDOW = 8;
constexpr uint64_t RESTART_SLOT_BYTES = 8ull << 30;   // memory for the window slots of one restart
struct RestartWalk {
  uint32_t count;          // diffs in this window
  int dense;               // node_list holds every chunk's NodeID (an earlier window wrote it)
  int last;                // no window follows (node_list is not written back)
  uint32_t main_cur;       // main diff's id: chunks it does not name start at (leaf, main_cur - 1)
  uint32_t n, N, cs;
  uint8_t* out;
  uint64_t out_len;
  uint2* node_list;
  const uint8_t* mflag;
  DevStatus* st;
  uint32_t width, per, per_log2;
  const uint8_t* data[RESTART_WINDOW];      // data sections
  uint64_t data_len[RESTART_WINDOW];        // bytes in each data section
  uint64_t datalen[RESTART_WINDOW];         // each header's datalen
  uint32_t cur[RESTART_WINDOW];             // each header's chkpt_id
  RestartSlot slot[RESTART_WINDOW];
};

// The one first-occurrence region (if any) whose root spans two leaf depths (chunk count not a
// power of two), found on the device after the region offsets are known.
struct StraddleInfo {
  int present;
  uint32_t root, region_off, lo, hi;
};
// roots that can span two depths: the common ancestors of the last inner node (n-2) and the
// first leaf of level D-1 (n-1), computed on the host from n alone
struct StraddleQuery {
  uint32_t count;
  uint32_t anc[32];
};
StraddleQuery straddle_query(uint32_t n);

// fills a.cum (device) from the repeat table of the device-resident diff a.diff
cudaError_t launch_restart_cum(const RestartArgs& a, cudaStream_t s);
// Expands one diff: clears the flags of a.slot (for the main diff also a.mflag), fills the
// slot, and for the main diff fills node_list and copies the chunks it resolves itself.  `sd`
// is device memory for the straddling-region record of this diff.
cudaError_t launch_restart_diff(const RestartArgs& a, StraddleInfo* sd, int sm_count, cudaStream_t s);
// resolves the chunks owed by the window's diffs and copies them
cudaError_t launch_restart_walk(const RestartWalk& w, int sm_count, cudaStream_t s);
// kernel launches made by one launch_restart_diff call (a walk is one launch)
int restart_diff_launches(uint32_t n, bool list);

}  // namespace b2d
