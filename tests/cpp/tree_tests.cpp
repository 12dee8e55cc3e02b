// C++ port of the reference's tree tests against the drop-in header (b200dedup_tree.hpp):
//   case <step0> <step1> <first> <shift> : test/test_case_NN.cpp -- chunk size 1, baseline +
//        one incremental checkpoint, restart both, check num_first_ocur()/num_shift_dupl()
//   tree_chkpt <chunk_size> <num_chkpts>  : test/tree_chkpt.cpp -- 1 MiB of fresh random bytes
//        per checkpoint, restart every checkpoint and compare
//   batch <count>                         : CheckpointBatch against one-at-a-time checkpoints
// Exit status 0 = pass, like the reference's ctest executables.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "b200dedup_tree.hpp"

static uint8_t* dev_copy(const std::vector<uint8_t>& h) {
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, h.size()) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice);
  return d;
}

static std::vector<uint8_t> host_copy(const uint8_t* d, size_t n) {
  std::vector<uint8_t> h(n);
  cudaMemcpy(h.data(), d, n, cudaMemcpyDeviceToHost);
  return h;
}

static int run_case(const char* s0, const char* s1, size_t first, size_t shift) {
  std::vector<uint8_t> a(s0, s0 + strlen(s0)), b(s1, s1 + strlen(s1));
  uint8_t* da = dev_copy(a);
  uint8_t* db = dev_copy(b);
  uint8_t* out = nullptr;
  cudaMalloc(&out, a.size());
  b2d::TreeDeduplicator dedup(1);
  std::vector<std::vector<uint8_t>> chkpts(1);
  std::string null("/dev/null/");
  dedup.checkpoint(da, a.size(), chkpts[0], true);
  dedup.restart(out, a.size(), chkpts, null, 0);
  if (host_copy(out, a.size()) != a) {
    printf("checkpoint 0 restart mismatch\n");
    return 1;
  }
  chkpts.emplace_back();
  dedup.checkpoint(db, b.size(), chkpts[1], false);
  dedup.restart(out, b.size(), chkpts, null, 1);
  if (host_copy(out, b.size()) != b) {
    printf("checkpoint 1 restart mismatch\n");
    return 1;
  }
  printf("Expected %zu first occurrence regions and %zu shifted duplicate regions\n", first, shift);
  printf("Found %zu first occurrence regions and %zu shifted duplicate regions\n", dedup.num_first_ocur(),
         dedup.num_shift_dupl());
  cudaFree(da);
  cudaFree(db);
  cudaFree(out);
  return (dedup.num_first_ocur() == first && dedup.num_shift_dupl() == shift) ? 0 : 1;
}

// tree_chkpt / list_chkpt (test/tree_chkpt.cpp, test/list_chkpt.cpp): random 1 MiB checkpoints,
// each restarted from the diffs so far and compared with the data
static int run_tree_chkpt(uint32_t chunk_size, uint32_t num_chkpts, bool list = false) {
  const size_t len = 1024 * 1024;
  std::mt19937_64 rng(1931);
  std::unique_ptr<b2d::TreeDeduplicator> owner(list ? new b2d::ListDeduplicator(chunk_size)
                                                    : new b2d::TreeDeduplicator(chunk_size));
  b2d::TreeDeduplicator& dedup = *owner;
  std::vector<std::vector<uint8_t>> chkpts;
  std::string null("/dev/null/");
  uint8_t* d = nullptr;
  uint8_t* out = nullptr;
  cudaMalloc(&d, len);
  cudaMalloc(&out, len);
  for (uint32_t i = 0; i < num_chkpts; i++) {
    std::vector<uint8_t> h(len);
    for (auto& x : h) x = (uint8_t)(rng() & 0xff);
    cudaMemcpy(d, h.data(), len, cudaMemcpyHostToDevice);
    chkpts.emplace_back();
    dedup.checkpoint(d, len, chkpts.back(), i == 0);
    dedup.restart(out, len, chkpts, null, i);
    if (host_copy(out, len) != h) {
      printf("Checkpoint %u\nHashes don't match!\n", i);
      return 1;
    }
    printf("Checkpoint %u\nHashes match!\n", i);
  }
  cudaFree(d);
  cudaFree(out);
  return 0;
}

// batch <count> : `count` buffers of uneven sizes, 3 checkpoints through a CheckpointBatch and
// through separate deduplicators one at a time; every diff must be equal
static int run_batch(uint32_t count) {
  std::mt19937_64 rng(7);
  std::vector<size_t> len;
  std::vector<std::vector<uint8_t>> host;
  std::vector<uint8_t*> dev;
  for (uint32_t i = 0; i < count; i++) {
    len.push_back(4096 + (size_t)(rng() % (1u << 20)));
    host.emplace_back(len.back());
    for (auto& x : host.back()) x = (uint8_t)(rng() & 0xff);
    dev.push_back(dev_copy(host.back()));
  }
  std::vector<b2d::TreeDeduplicator*> batched, alone;
  for (uint32_t i = 0; i < count; i++) {
    batched.push_back(new b2d::TreeDeduplicator(128));
    alone.push_back(new b2d::TreeDeduplicator(128));
  }
  b2d::CheckpointBatch batch;
  int rc = 0;
  for (int c = 0; c < 3 && rc == 0; c++) {
    if (c > 0)
      for (uint32_t i = 0; i < count; i++) {   // rewrite a few chunks of every buffer
        for (size_t k = 0; k < 64 && k < host[i].size(); k++) host[i][(rng() % host[i].size())] ^= 0x5a;
        cudaMemcpy(dev[i], host[i].data(), len[i], cudaMemcpyHostToDevice);
      }
    batch.checkpoint(batched, dev, len);
    for (uint32_t i = 0; i < count; i++) {
      std::vector<uint8_t> want;
      alone[i]->checkpoint(dev[i], len[i], want, c == 0);
      if (b2d::diff(*batched[i]) != want) {
        printf("batch checkpoint %d buffer %u differs\n", c, i);
        rc = 1;
      }
    }
  }
  for (uint32_t i = 0; i < count; i++) {
    delete batched[i];
    delete alone[i];
    cudaFree(dev[i]);
  }
  if (rc == 0) printf("batch of %u: all diffs equal\n", count);
  return rc;
}

int main(int argc, char** argv) {
  try {
    if (argc == 6 && std::string(argv[1]) == "case")
      return run_case(argv[2], argv[3], strtoull(argv[4], nullptr, 10), strtoull(argv[5], nullptr, 10));
    if (argc == 4 && std::string(argv[1]) == "tree_chkpt")
      return run_tree_chkpt((uint32_t)atoi(argv[2]), (uint32_t)atoi(argv[3]));
    if (argc == 4 && std::string(argv[1]) == "list_chkpt")
      return run_tree_chkpt((uint32_t)atoi(argv[2]), (uint32_t)atoi(argv[3]), true);
    if (argc == 3 && std::string(argv[1]) == "batch") return run_batch((uint32_t)atoi(argv[2]));
  } catch (const b2d::Error& e) {
    printf("error: %s\n", e.what());
    return 2;
  }
  printf("usage: tree_tests case <step0> <step1> <first> <shift> | tree_chkpt <chunk_size> <num_chkpts>\n");
  return 64;
}
