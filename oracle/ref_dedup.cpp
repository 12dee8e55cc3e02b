// C entry points over the reference's own TreeDeduplicator and ListDeduplicator
// (src/tree_approach.cpp, src/list_approach.cpp, compiled unmodified where they lie against the
// sequential Kokkos stand-in in oracle/kokkos_shim/).  TEST INFRASTRUCTURE ONLY: built into
// oracle/_ref/libref_dedup.so by oracle/Makefile when the reference source tree is present;
// tests/golden/make_golden.py and the CPU tests use it to pin the oracle's diff bytes to the
// reference's own code.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "list_approach.hpp"
#include "tree_approach.hpp"

using Host = Kokkos::View<uint8_t*>::HostMirror;

namespace {

template <class Dedup>
int checkpoint_with(Dedup* t, const uint8_t* data, uint64_t len, int make_baseline, uint8_t** out,
                    uint64_t* out_len) {
  Host diff_h("Diff", 1);
  t->checkpoint(const_cast<uint8_t*>(data), len, diff_h, make_baseline != 0);
  *out_len = diff_h.size();
  *out = static_cast<uint8_t*>(std::malloc(diff_h.size() ? diff_h.size() : 1));
  if (!*out) return -1;
  std::memcpy(*out, diff_h.data(), diff_h.size());
  return 0;
}

template <class Dedup>
int restart_with(uint32_t chunk_size, const uint8_t* const* diffs, const uint64_t* sizes, uint32_t count,
                 uint32_t chkpt_id, uint8_t* out, uint64_t out_len) {
  Dedup t(chunk_size);
  std::vector<Host> chkpts;
  for (uint32_t i = 0; i < count; i++) {
    Host h("Checkpoint", sizes[i]);
    std::memcpy(h.data(), diffs[i], sizes[i]);
    chkpts.push_back(h);
  }
  Kokkos::View<uint8_t*> data("Restart", out_len);
  std::memcpy(data.data(), out, out_len);
  std::string logname = "/dev/null";   // the restart log cannot be opened there and is skipped
  t.restart(data, chkpts, logname, chkpt_id);
  std::memcpy(out, data.data(), out_len);
  return 0;
}

}  // namespace

extern "C" {

void* ref_tree_create(uint32_t chunk_size) { return new TreeDeduplicator(chunk_size); }
void ref_tree_destroy(void* d) { delete static_cast<TreeDeduplicator*>(d); }
// checkpoint(data_ptr, len, diff_h, make_baseline) -- src/tree_approach.cpp:1740-1748; the diff
// is returned in malloc'd memory (free with ref_free)
int ref_tree_checkpoint(void* d, const uint8_t* data, uint64_t len, int make_baseline, uint8_t** out,
                        uint64_t* out_len) {
  return checkpoint_with(static_cast<TreeDeduplicator*>(d), data, len, make_baseline, out, out_len);
}
uint64_t ref_tree_num_first_ocur(void* d) { return static_cast<TreeDeduplicator*>(d)->num_first_ocur(); }
uint64_t ref_tree_num_shift_dupl(void* d) { return static_cast<TreeDeduplicator*>(d)->num_shift_dupl(); }
// restart(View data, vector<HostMirror>& chkpts, logname, chkpt_id) -- src/tree_approach.cpp:1786-1817,
// into `out` (out_len bytes, which the caller initialises)
int ref_tree_restart(uint32_t chunk_size, const uint8_t* const* diffs, const uint64_t* sizes, uint32_t count,
                     uint32_t chkpt_id, uint8_t* out, uint64_t out_len) {
  return restart_with<TreeDeduplicator>(chunk_size, diffs, sizes, count, chkpt_id, out, out_len);
}

void* ref_list_create(uint32_t chunk_size) { return new ListDeduplicator(chunk_size); }
void ref_list_destroy(void* d) { delete static_cast<ListDeduplicator*>(d); }
// the same overloads of the list approach (src/list_approach.cpp)
int ref_list_checkpoint(void* d, const uint8_t* data, uint64_t len, int make_baseline, uint8_t** out,
                        uint64_t* out_len) {
  return checkpoint_with(static_cast<ListDeduplicator*>(d), data, len, make_baseline, out, out_len);
}
int ref_list_restart(uint32_t chunk_size, const uint8_t* const* diffs, const uint64_t* sizes, uint32_t count,
                     uint32_t chkpt_id, uint8_t* out, uint64_t out_len) {
  return restart_with<ListDeduplicator>(chunk_size, diffs, sizes, count, chkpt_id, out, out_len);
}

void ref_free(void* p) { std::free(p); }

}  // extern "C"
