// dedup_files: deduplicate a sequence of checkpoint files with the B200 deduplicators.
//
// Command line of the reference's driver (src/dedup_files.cpp:10-21, argv layout :30-48):
//   dedup_files chunk_size num_chkpts --run-tree-chkpt|--run-list-chkpt file_0 ... file_{num_chkpts-1}
// Each file is loaded into device memory and checkpointed in order (file_0 as the baseline);
// the diff is written next to it as <file>.hashtree.incr_chkpt (tree) or
// <file>.hashlist.incr_chkpt (list), and the reference's per-checkpoint log under the file's
// base name (src/dedup_files.cpp:88-102).  The tree and list approaches are built here; the
// reference's full and basic approaches are rejected.
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

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s chunk_size num_chkpts --run-tree-chkpt|--run-list-chkpt file...\n", argv[0]);
    return 1;
  }
  const uint32_t chunk_size = (uint32_t)std::strtoul(argv[1], nullptr, 10);
  const uint32_t num_chkpts = (uint32_t)std::strtoul(argv[2], nullptr, 10);
  const bool list = std::strcmp(argv[3], "--run-list-chkpt") == 0;
  if (!list && std::strcmp(argv[3], "--run-tree-chkpt") != 0) {
    std::fprintf(stderr, "error: mode %s is not built here; only --run-tree-chkpt and --run-list-chkpt\n", argv[3]);
    return 2;
  }
  if (chunk_size == 0 || (uint32_t)argc < 4 + num_chkpts) {
    std::fprintf(stderr, "error: expected chunk_size > 0 and %u checkpoint files\n", num_chkpts);
    return 1;
  }
  try {
    std::unique_ptr<b2d::TreeDeduplicator> owner(list ? new b2d::ListDeduplicator(chunk_size)
                                                      : new b2d::TreeDeduplicator(chunk_size));
    b2d::TreeDeduplicator& dedup = *owner;
    std::vector<uint8_t> host;
    uint8_t* dev = nullptr;
    size_t cap = 0;
    for (uint32_t idx = 0; idx < num_chkpts; idx++) {
      const std::string path = argv[4 + idx];
      if (!read_file(path, host)) {
        std::fprintf(stderr, "error: cannot read %s\n", path.c_str());
        return 3;
      }
      if (host.size() > cap) {
        if (dev) cudaFree(dev);
        cap = host.size();
        if (cudaMalloc(&dev, cap) != cudaSuccess) {
          std::fprintf(stderr, "error: cannot allocate %zu device bytes\n", cap);
          return 4;
        }
      }
      if (cudaMemcpy(dev, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) return 4;
      std::string filename = path + (list ? ".hashlist.incr_chkpt" : ".hashtree.incr_chkpt");
      std::string logname = path.substr(path.rfind('/') + 1);
      dedup.checkpoint(dev, host.size(), filename, logname, idx == 0);
      std::printf("checkpoint %u: %s -> %s (first regions %zu, shifted regions %zu)\n", idx, path.c_str(),
                  filename.c_str(), dedup.num_first_ocur(), dedup.num_shift_dupl());
    }
    if (dev) cudaFree(dev);
  } catch (const b2d::Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 5;
  }
  return 0;
}
