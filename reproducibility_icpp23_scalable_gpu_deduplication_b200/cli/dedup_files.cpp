// dedup_files: deduplicate a sequence of checkpoint files with the B200 deduplicators.
//
// Command line of the reference's driver (src/dedup_files.cpp:10-21, argv layout :30-48):
//   dedup_files chunk_size num_chkpts --run-tree-chkpt|--run-list-chkpt file_0 ... file_{num_chkpts-1}
// Each file is loaded into device memory and checkpointed in order (file_0 as the baseline);
// the diff is written next to it as <file>.hashtree.incr_chkpt (tree) or
// <file>.hashlist.incr_chkpt (list), and the reference's per-checkpoint log under the file's
// base name (src/dedup_files.cpp:88-102).  The tree and list approaches are built here; the
// reference's full and basic approaches are rejected.
//
// The file I/O overlaps the GPU work: while checkpoint i runs, a reader thread loads file i+1
// into page-locked memory and a writer thread writes diff i-1; diff i is copied back
// asynchronously into one of two page-locked buffers (the next checkpoint's kernels queue
// behind that copy on the same stream).  The reference does these steps one after another
// (its timers[3] is the copy-back); the files and logs written are the same, with the log's
// Write Time column 0 since the copy-back is no longer inside the checkpoint.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <memory>
#include <string>
#include <vector>

#include "b200dedup_tree.hpp"

// bytes in page-locked host memory, grown as needed
struct PinnedBlock {
  uint8_t* p = nullptr;
  size_t cap = 0, len = 0;
  PinnedBlock() = default;
  PinnedBlock(const PinnedBlock&) = delete;
  PinnedBlock& operator=(const PinnedBlock&) = delete;
  ~PinnedBlock() {
    if (p) cudaFreeHost(p);
  }
  bool reserve(size_t n) {
    if (p && n <= cap) return true;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    if (cudaMallocHost(reinterpret_cast<void**>(&p), n ? n : 1) != cudaSuccess) {
      p = nullptr;
      return false;
    }
    cap = n ? n : 1;
    return true;
  }
};

static bool read_into(const std::string& path, PinnedBlock* b) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  bool ok = std::fseek(f, 0, SEEK_END) == 0;
  const long n = ok ? std::ftell(f) : -1;
  ok = ok && n >= 0 && std::fseek(f, 0, SEEK_SET) == 0 && b->reserve((size_t)n);
  if (ok) {
    b->len = (size_t)n;
    ok = n == 0 || std::fread(b->p, 1, (size_t)n, f) == (size_t)n;
  }
  std::fclose(f);
  return ok;
}

static bool write_from(const std::string& path, const uint8_t* p, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = n == 0 || std::fwrite(p, 1, n, f) == n;
  return (std::fclose(f) == 0) && ok;
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
  int rc = 0;
  uint8_t* dev = nullptr;
  size_t dev_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr};
  PinnedBlock in[2], out[2];
  std::future<bool> reading, writing[2];
  std::string written[2];
  try {
    std::unique_ptr<b2d::TreeDeduplicator> owner(list ? new b2d::ListDeduplicator(chunk_size)
                                                      : new b2d::TreeDeduplicator(chunk_size));
    b2d_dedup* h = owner->handle();
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&copied[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&copied[1], cudaEventDisableTiming) != cudaSuccess) {
      std::fprintf(stderr, "error: cannot create a CUDA stream or event\n");
      return 4;
    }
    b2d::check(b2d_set_stream(h, stream), "set_stream");
    if (num_chkpts) reading = std::async(std::launch::async, read_into, std::string(argv[4]), &in[0]);
    for (uint32_t idx = 0; idx < num_chkpts && rc == 0; idx++) {
      const std::string path = argv[4 + idx];
      PinnedBlock& cur = in[idx % 2];
      if (!reading.get()) {
        std::fprintf(stderr, "error: cannot read %s\n", path.c_str());
        rc = 3;
        break;
      }
      // the other input buffer fed checkpoint idx-1, which has completed
      if (idx + 1 < num_chkpts)
        reading = std::async(std::launch::async, read_into, std::string(argv[5 + idx]), &in[(idx + 1) % 2]);
      if (cur.len > dev_cap) {
        cudaStreamSynchronize(stream);
        if (dev) cudaFree(dev);
        dev = nullptr;
        dev_cap = 0;
        if (cudaMalloc(reinterpret_cast<void**>(&dev), cur.len) != cudaSuccess) {
          std::fprintf(stderr, "error: cannot allocate %zu device bytes\n", cur.len);
          rc = 4;
          break;
        }
        dev_cap = cur.len;
      }
      if (cudaMemcpyAsync(dev, cur.p, cur.len, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
        rc = 4;
        break;
      }
      // checkpoint(.., filename, logname, make_baseline) (:1705-1724) with the diff left on the device
      uint64_t dlen = 0;
      b2d::check(b2d_checkpoint_device(h, dev, cur.len, idx == 0, 1, &dlen), "checkpoint");
      const std::string logname = path.substr(path.rfind('/') + 1);
      b2d::check(b2d_write_chkpt_log(h, logname.c_str()), "checkpoint log");
      const uint32_t k = idx % 2;
      if (writing[k].valid() && !writing[k].get()) {   // diff idx-2 is on disk; its buffer is free
        std::fprintf(stderr, "error: cannot write %s\n", written[k].c_str());
        rc = 3;
        break;
      }
      if (!out[k].reserve(dlen)) {
        std::fprintf(stderr, "error: cannot allocate %llu page-locked bytes\n", (unsigned long long)dlen);
        rc = 4;
        break;
      }
      b2d::check(b2d_copy_diff_async(h, out[k].p, out[k].cap, stream), "copy diff");
      if (cudaEventRecord(copied[k], stream) != cudaSuccess) {
        rc = 4;
        break;
      }
      written[k] = path + (list ? ".hashlist.incr_chkpt" : ".hashtree.incr_chkpt");
      const std::string fname = written[k];
      const uint8_t* src = out[k].p;
      const cudaEvent_t ev = copied[k];
      writing[k] = std::async(std::launch::async, [fname, src, dlen, ev] {
        return cudaEventSynchronize(ev) == cudaSuccess && write_from(fname, src, (size_t)dlen);
      });
      std::printf("checkpoint %u: %s -> %s (first regions %zu, shifted regions %zu)\n", idx, path.c_str(),
                  written[k].c_str(), owner->num_first_ocur(), owner->num_shift_dupl());
    }
    for (int k = 0; k < 2; k++)
      if (writing[k].valid() && !writing[k].get() && rc == 0) {
        std::fprintf(stderr, "error: cannot write %s\n", written[k].c_str());
        rc = 3;
      }
    if (reading.valid()) reading.wait();
  } catch (const b2d::Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    rc = 5;
  }
  for (int k = 0; k < 2; k++)
    if (writing[k].valid()) writing[k].wait();
  if (reading.valid()) reading.wait();
  if (stream) cudaStreamSynchronize(stream);
  if (dev) cudaFree(dev);
  for (auto& e : copied)
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
  return rc;
}
