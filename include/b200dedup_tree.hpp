// b200dedup_tree.hpp -- header-only C++ mirror of the reference's TreeDeduplicator over the
// C ABI in b200dedup.h.
//
// Same method set and argument meaning as include/tree_approach.hpp:16-205 and
// include/deduplicator_interface.hpp:14-184 of TauferLab/Reproducibility_ICPP23_Scalable_GPU_
// Deduplication, with the Kokkos types replaced:
//   Kokkos::View<uint8_t*>::HostMirror  -> std::vector<uint8_t>   (a diff on the host)
//   Kokkos::View<uint8_t*> (device)     -> uint8_t* device pointer + length
// Errors become b2d::Error exceptions on this side of the boundary (the C ABI itself returns
// status codes).  Link against libb200dedup.so.
#ifndef B200DEDUP_TREE_HPP
#define B200DEDUP_TREE_HPP

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "b200dedup.h"

namespace b2d {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what)
      : std::runtime_error(what + ": " + b2d_strerror(code)), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* what) {
  if (rc != B2D_OK) throw Error(rc, what);
}

// header_t, include/utils.hpp:29-37
struct header_t {
  uint32_t ref_id;
  uint32_t chkpt_id;
  uint64_t datalen;
  uint32_t chunk_size;
  uint32_t num_first_ocur;
  uint32_t num_prior_chkpts;
  uint32_t num_shift_dupl;
};
static_assert(sizeof(header_t) == 32, "header_t is 32 bytes");

class TreeDeduplicator {
 public:
  explicit TreeDeduplicator(uint32_t bytes_per_chunk, int hash_kind = B2D_HASH_MURMUR3) {
    check(b2d_create(bytes_per_chunk, hash_kind, &h_), "TreeDeduplicator");
  }
  virtual ~TreeDeduplicator() {
    if (h_) b2d_destroy(h_);
  }
  TreeDeduplicator(const TreeDeduplicator&) = delete;
  TreeDeduplicator& operator=(const TreeDeduplicator&) = delete;

  // checkpoint(header_t&, uint8_t*, size_t, HostMirror&, bool)  (tree_approach.cpp:1577);
  // like the reference overload, it does not advance current_id
  void checkpoint(header_t& header, uint8_t* data_ptr, size_t data_len, std::vector<uint8_t>& diff_h,
                  bool make_baseline) {
    uint64_t n = 0;
    check(b2d_checkpoint_device(h_, data_ptr, data_len, make_baseline, 0, &n), "checkpoint");
    diff_h.resize(n);
    check(b2d_copy_diff(h_, diff_h.data(), n), "checkpoint");
    std::memcpy(&header, diff_h.data(), sizeof(header_t));
  }
  // checkpoint(uint8_t*, size_t, std::string& filename, std::string& logname, bool)  (:1705)
  void checkpoint(uint8_t* data_ptr, size_t len, std::string& filename, std::string& logname, bool make_baseline) {
    check(b2d_checkpoint_file(h_, data_ptr, len, filename.c_str(), logname.c_str(), make_baseline), "checkpoint");
  }
  // checkpoint(uint8_t*, size_t, HostMirror& diff_h, bool)  (:1740)
  void checkpoint(uint8_t* data_ptr, size_t len, std::vector<uint8_t>& diff_h, bool make_baseline) {
    const uint8_t* p = nullptr;
    uint64_t n = 0;
    check(b2d_checkpoint(h_, data_ptr, len, make_baseline, &p, &n), "checkpoint");
    diff_h.assign(p, p + n);
  }
  // checkpoint(uint8_t*, size_t, HostMirror& diff_h, std::string& logname, bool)  (:1765)
  void checkpoint(uint8_t* data_ptr, size_t len, std::vector<uint8_t>& diff_h, std::string& logname,
                  bool make_baseline) {
    const uint8_t* p = nullptr;
    uint64_t n = 0;
    check(b2d_checkpoint_log(h_, data_ptr, len, logname.c_str(), make_baseline, &p, &n), "checkpoint");
    diff_h.assign(p, p + n);
  }

  // restart(uint8_t* data_ptr, size_t len, vector<HostMirror>& chkpts, std::string& logname, id)  (:1807)
  void restart(uint8_t* data_ptr, size_t len, std::vector<std::vector<uint8_t>>& chkpts, std::string& logname,
               uint32_t chkpt_id) {
    std::vector<const uint8_t*> ptrs;
    std::vector<uint64_t> sizes;
    for (auto& c : chkpts) {
      ptrs.push_back(c.data());
      sizes.push_back(c.size());
    }
    check(b2d_restart(h_, data_ptr, len, ptrs.data(), sizes.data(), (uint32_t)chkpts.size(), chkpt_id,
                      logname.c_str()),
          "restart");
  }
  // restart(View data, vector<string>& chkpt_filenames, std::string& logname, id)  (:1827)
  void restart(uint8_t* data_ptr, size_t len, std::vector<std::string>& chkpt_filenames, std::string& logname,
               uint32_t chkpt_id) {
    std::vector<const char*> names;
    for (auto& s : chkpt_filenames) names.push_back(s.c_str());
    check(b2d_restart_files(h_, data_ptr, len, names.data(), (uint32_t)names.size(), chkpt_id, logname.c_str()),
          "restart");
  }

  // write_chkpt_log(header_t&, HostMirror& diff_h, std::string& logname)
  // (deduplicator_interface.hpp:172-174): the three CSV logs, Chkpt ID = current_id()
  void write_chkpt_log(header_t& header, std::vector<uint8_t>& diff_h, std::string& logname) {
    check(b2d_write_chkpt_log_host(h_, &header, diff_h.data(), diff_h.size(), logname.c_str()), "write_chkpt_log");
  }
  // write_restart_log(uint32_t select_chkpt, std::string& logname)  (deduplicator_interface.hpp:181-182)
  void write_restart_log(uint32_t select_chkpt, std::string& logname) {
    check(b2d_write_restart_log(h_, select_chkpt, logname.c_str()), "write_restart_log");
  }

  size_t num_first_ocur() {
    uint64_t v = 0;
    check(b2d_num_first_ocur(h_, &v), "num_first_ocur");
    return v;
  }
  size_t num_shift_dupl() {
    uint64_t v = 0;
    check(b2d_num_shift_dupl(h_, &v), "num_shift_dupl");
    return v;
  }
  uint32_t current_id() {
    uint32_t v = 0;
    check(b2d_current_id(h_, &v), "current_id");
    return v;
  }
  std::pair<uint64_t, uint64_t> datasizes() {
    uint64_t v[2] = {0, 0};
    check(b2d_datasizes(h_, v), "datasizes");
    return {v[0], v[1]};
  }
  b2d_dedup* handle() { return h_; }

 protected:
  struct ListTag {};
  TreeDeduplicator(uint32_t bytes_per_chunk, int hash_kind, ListTag) {
    check(b2d_create_list(bytes_per_chunk, hash_kind, &h_), "ListDeduplicator");
  }

 private:
  b2d_dedup* h_ = nullptr;
};

// ListDeduplicator(uint32_t bytes_per_chunk) -- src/list_approach.cpp:5-9, with the same method
// set (include/list_approach.hpp): checkpoint overloads write list diffs naming chunk indices,
// restarts take list diffs.  Batches take list handles beside tree handles.
class ListDeduplicator : public TreeDeduplicator {
 public:
  explicit ListDeduplicator(uint32_t bytes_per_chunk, int hash_kind = B2D_HASH_MURMUR3)
      : TreeDeduplicator(bytes_per_chunk, hash_kind, ListTag{}) {}
};

// Batched checkpoints (b2d_batch_*): one checkpoint of each of many TreeDeduplicators' buffers
// per call, sharing launches; each deduplicator's result is what its own checkpoint gives.
// No reference counterpart.
class CheckpointBatch {
 public:
  CheckpointBatch() { check(b2d_batch_create(&b_), "CheckpointBatch"); }
  ~CheckpointBatch() {
    if (b_) b2d_batch_destroy(b_);
  }
  CheckpointBatch(const CheckpointBatch&) = delete;
  CheckpointBatch& operator=(const CheckpointBatch&) = delete;

  void set_param(const char* name, int64_t value) { check(b2d_batch_set_param(b_, name, value), name); }
  // checkpoint device buffers data[i] (len[i] bytes) through dedups[i]; make_baseline may be
  // empty (no forced baselines).  Diffs are then read per deduplicator (diff()).
  void checkpoint(std::vector<TreeDeduplicator*>& dedups, const std::vector<uint8_t*>& data,
                  const std::vector<size_t>& len, const std::vector<int>& make_baseline = {}) {
    std::vector<b2d_dedup*> hs;
    std::vector<const void*> ptrs;
    std::vector<uint64_t> lens;
    for (size_t i = 0; i < dedups.size(); i++) {
      hs.push_back(dedups[i]->handle());
      ptrs.push_back(data[i]);
      lens.push_back(len[i]);
    }
    std::vector<int> rcs(dedups.size(), 0);
    check(b2d_batch_checkpoint(b_, hs.data(), ptrs.data(), lens.data(),
                               make_baseline.empty() ? nullptr : make_baseline.data(), (uint32_t)hs.size(),
                               rcs.data()),
          "batch checkpoint");
  }

 private:
  b2d_batch* b_ = nullptr;
};

// the last diff of a deduplicator, copied to the host
inline std::vector<uint8_t> diff(TreeDeduplicator& d) {
  const void* p = nullptr;
  uint64_t n = 0;
  check(b2d_diff_device(d.handle(), &p, &n), "diff");
  std::vector<uint8_t> out(n);
  check(b2d_copy_diff(d.handle(), out.data(), n), "diff");
  return out;
}

}  // namespace b2d

#endif  // B200DEDUP_TREE_HPP
