// C++ port of the reference's tree tests against the drop-in header (b200dedup_tree.hpp):
//   case <step0> <step1> <first> <shift> : test/test_case_NN.cpp -- chunk size 1, baseline +
//        one incremental checkpoint, restart both, check num_first_ocur()/num_shift_dupl()
//   tree_chkpt <chunk_size> <num_chkpts>  : test/tree_chkpt.cpp -- 1 MiB of fresh random bytes
//        per checkpoint, restart every checkpoint and compare
// Exit status 0 = pass, like the reference's ctest executables.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
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

static int run_tree_chkpt(uint32_t chunk_size, uint32_t num_chkpts) {
  const size_t len = 1024 * 1024;
  std::mt19937_64 rng(1931);
  b2d::TreeDeduplicator dedup(chunk_size);
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

int main(int argc, char** argv) {
  try {
    if (argc == 6 && std::string(argv[1]) == "case")
      return run_case(argv[2], argv[3], strtoull(argv[4], nullptr, 10), strtoull(argv[5], nullptr, 10));
    if (argc == 4 && std::string(argv[1]) == "tree_chkpt")
      return run_tree_chkpt((uint32_t)atoi(argv[2]), (uint32_t)atoi(argv[3]));
  } catch (const b2d::Error& e) {
    printf("error: %s\n", e.what());
    return 2;
  }
  printf("usage: tree_tests case <step0> <step1> <first> <shift> | tree_chkpt <chunk_size> <num_chkpts>\n");
  return 64;
}
