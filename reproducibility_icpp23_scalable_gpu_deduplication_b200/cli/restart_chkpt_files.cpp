// restart_chkpt_files: rebuild one checkpoint from <file>.hashtree.incr_chkpt (tree) or
// <file>.hashlist.incr_chkpt (list) diffs.
//
// Command line of the reference's driver (src/restart_chkpt_files.cpp:26-45):
//   restart_chkpt_files restart_id num_chkpts num_tests chunk_size --run-tree-chkpt|--run-list-chkpt file...
// `file_i` are the original checkpoint files (their sizes give the restart length, :72-77);
// the diffs are read from file_i.hashtree.incr_chkpt (:57-60, :171-184) or
// file_i.hashlist.incr_chkpt (:53-56, :140-151).  Checkpoint
// `restart_id` is rebuilt `num_tests` times into device memory and its digest printed the way
// the reference does (:188-195, include/hash_functions.hpp:47-63: the chunk hash of the whole
// buffer, upper-case hex, a space after every 4 bytes).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "b200dedup_tree.hpp"

static bool read_file(const std::string& path, std::vector<uint8_t>& out) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return false;
  const std::streamsize n = f.tellg();
  f.seekg(0);
  out.resize((size_t)n);
  return n == 0 || (bool)f.read(reinterpret_cast<char*>(out.data()), n);
}

static long file_size(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  return f ? (long)f.tellg() : -1;
}

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr,
                 "usage: %s restart_id num_chkpts num_tests chunk_size --run-tree-chkpt|--run-list-chkpt file...\n",
                 argv[0]);
    return 1;
  }
  const uint32_t restart_id = (uint32_t)std::strtoul(argv[1], nullptr, 10);
  const uint32_t num_chkpts = (uint32_t)std::strtoul(argv[2], nullptr, 10);
  const uint32_t num_tests = (uint32_t)std::strtoul(argv[3], nullptr, 10);
  const uint32_t chunk_size = (uint32_t)std::strtoul(argv[4], nullptr, 10);
  const bool list = std::strcmp(argv[5], "--run-list-chkpt") == 0;
  if (!list && std::strcmp(argv[5], "--run-tree-chkpt") != 0) {
    std::fprintf(stderr, "error: mode %s is not built here; only --run-tree-chkpt and --run-list-chkpt\n", argv[5]);
    return 2;
  }
  const std::string suffix = list ? ".hashlist.incr_chkpt" : ".hashtree.incr_chkpt";
  if (chunk_size == 0 || restart_id >= num_chkpts || (uint32_t)argc < 6 + num_chkpts) {
    std::fprintf(stderr, "error: expected chunk_size > 0, restart_id < num_chkpts and %u files\n", num_chkpts);
    return 1;
  }
  std::vector<std::string> files;
  for (uint32_t i = 0; i < num_chkpts; i++) files.push_back(argv[6 + i]);
  const long len = file_size(files[restart_id]);
  if (len <= 0) {
    std::fprintf(stderr, "error: cannot read %s\n", files[restart_id].c_str());
    return 3;
  }
  std::vector<std::vector<uint8_t>> diffs(num_chkpts);
  for (uint32_t i = 0; i < num_chkpts; i++) {
    if (!read_file(files[i] + suffix, diffs[i])) {
      std::fprintf(stderr, "error: cannot read %s%s\n", files[i].c_str(), suffix.c_str());
      return 3;
    }
  }
  uint8_t* dev = nullptr;
  if (cudaMalloc(&dev, (size_t)len) != cudaSuccess) {
    std::fprintf(stderr, "error: cannot allocate %ld device bytes\n", len);
    return 4;
  }
  std::vector<uint8_t> host((size_t)len);
  int rc = 0;
  try {
    for (uint32_t t = 0; t < num_tests; t++) {
      cudaMemset(dev, 0, (size_t)len);
      std::unique_ptr<b2d::TreeDeduplicator> owner(list ? new b2d::ListDeduplicator(chunk_size)
                                                        : new b2d::TreeDeduplicator(chunk_size));
      b2d::TreeDeduplicator& dedup = *owner;
      std::string logname = files[restart_id].substr(files[restart_id].rfind('/') + 1);
      dedup.restart(dev, (size_t)len, diffs, logname, restart_id);
      if (cudaMemcpy(host.data(), dev, (size_t)len, cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = 4;
        break;
      }
      uint8_t dg[16];
      b2d_hash_host(B2D_HASH_MURMUR3, host.data(), (uint64_t)len, dg);
      static const char hexchars[] = "0123456789ABCDEF";
      std::string s;
      for (int k = 0; k < 16; k++) {
        s += hexchars[dg[k] >> 4];
        s += hexchars[dg[k] & 0xF];
        if (k % 4 == 3) s += ' ';
      }
      std::printf(list ? "Hashlist digest:       %s\n" : "Hashtree digest:       %s\n", s.c_str());
    }
  } catch (const b2d::Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    rc = 5;
  }
  cudaFree(dev);
  return rc;
}
