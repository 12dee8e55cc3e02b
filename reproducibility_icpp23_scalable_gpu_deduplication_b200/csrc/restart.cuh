// Restart kernel arguments (see restart.cu).
#pragma once
#include "common.cuh"
#include "dedup_kernels.cuh"

namespace b2d {

// dist[] entries are u32 chunk offsets widened to u64, so the absent marker never collides
// with an offset (the reference computes some offsets in wrapping u32 arithmetic)
constexpr unsigned long long R_ABSENT = ~0ull;

struct RestartArgs {
  const uint8_t* diff;     // device copy of one diff (header at offset 0 of this pointer)
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
  uint2* node_list;        // n
  unsigned long long* dist;   // n
  uint2* rep;              // n
  const unsigned long long* cum;   // inclusive shift counts per checkpoint id (ncum entries)
  uint32_t ncum;
  uint32_t* offs;          // scratch: F or S exclusive offsets
  uint32_t* partial;       // SCAN_GRID
  unsigned long long* total;
  DevStatus* st;
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

cudaError_t launch_restart_init(const RestartArgs& a, int sm_count, cudaStream_t s);
// fills a.cum (device) from the repeat table of the device-resident diff a.diff
cudaError_t launch_restart_cum(const RestartArgs& a, cudaStream_t s);
// `sd` is device memory for the straddling-region record of this diff
cudaError_t launch_restart_diff(const RestartArgs& a, StraddleInfo* sd, int sm_count, cudaStream_t s);

}  // namespace b2d
