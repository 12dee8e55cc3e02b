/*
 * b200dedup.h -- C ABI of the B200 tree-approach incremental-checkpoint deduplicator.
 *
 * Drop-in for the reference's TreeDeduplicator (TauferLab/Reproducibility_ICPP23_Scalable_GPU_
 * Deduplication, include/tree_approach.hpp:16-205 over include/deduplicator_interface.hpp:
 * 14-184).  Plain pointers and sizes only; every call returns an int status (B2D_OK = 0,
 * negative on error, see b2d_strerror) and no C++ exception crosses this boundary.
 *
 * Diff format (".hashtree.incr_chkpt", little endian; src/tree_approach.cpp:777-780):
 *   header_t {u32 ref_id; u32 chkpt_id; u64 datalen; u32 chunk_size; u32 num_first_ocur;
 *             u32 num_prior_chkpts; u32 num_shift_dupl}                 (include/utils.hpp:29-37)
 *   u32 first-occurrence region root  x num_first_ocur
 *   (u32 checkpoint id, u32 count)    x num_prior_chkpts
 *   (u32 node, u32 source node)       x num_shift_dupl
 *   chunk data of the first-occurrence regions
 * The bytes are identical to the reference's output run sequentially (its parallel atomics
 * only permute them).
 *
 * Threading: one handle per host thread; a handle is not thread-safe.  All device work of a
 * handle runs on one CUDA stream (its own, or the one given to b2d_set_stream).  Device
 * pointers passed in must belong to the current device.
 */
#ifndef B200DEDUP_H
#define B200DEDUP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b2d_dedup b2d_dedup;

enum b2d_status {
  B2D_OK = 0,
  B2D_ERR_ARG = -1,            /* invalid argument */
  B2D_ERR_CUDA = -2,           /* a CUDA runtime call failed */
  B2D_ERR_NOMEM = -3,          /* device or host allocation failed */
  B2D_ERR_FORMAT = -4,         /* a diff is truncated or its header is inconsistent */
  B2D_ERR_IO = -5,             /* file open/read/write failed */
  B2D_ERR_MAP_FULL = -6,       /* digest map probe sequence exhausted (should not happen) */
  B2D_ERR_TIMEOUT = -7,        /* a bounded device wait gave up */
  B2D_ERR_INTERNAL = -8,       /* an invariant of the algorithm did not hold */
  B2D_ERR_RESTART_RANGE = -9,  /* restart met an index/offset outside its buffers (corrupt
                                  diff, or the reference's non-power-of-two region quirk);
                                  the offending copies were skipped */
  B2D_ERR_LEN_CHANGED = -10,   /* buffer length changed without make_baseline, or the handle
                                  holds no complete checkpoint (after a failed one) and this
                                  one is not a baseline */
  B2D_ERR_UNSUPPORTED = -11    /* outside the supported range: checkpoint ids (which, as in the
                                  reference, keep counting across baselines) up to 8190 per
                                  handle; a longer run continues on a new handle */
};

enum b2d_hash_kind {
  B2D_HASH_MURMUR3 = 0, /* reference default: include/hash_functions.hpp:19 */
  B2D_HASH_MD5 = 1      /* the commented alternative: include/hash_functions.hpp:18 */
};

/* TreeDeduplicator(uint32_t bytes_per_chunk) -- src/tree_approach.cpp:5-9.  The hash is a
 * compile-time choice in the reference (include/hash_functions.hpp:16-20); here a parameter. */
int b2d_create(uint32_t chunk_size, int hash_kind, b2d_dedup** out);
/* ListDeduplicator(uint32_t bytes_per_chunk) -- src/list_approach.cpp:5-9: the list approach
 * (one digest per chunk, a changed chunk is a first occurrence or a shifted duplicate,
 * src/list_approach.cpp:23-257) behind the same handle.  Every call below takes it: checkpoint
 * overloads (:843-974, diffs naming chunk indices), host and device restarts (:259-586), file
 * and log forms ("List" rows), and batches (alone or mixed with tree handles; a list handle
 * labels and assembles its diff in its own branch of the batch).  Not by b2d_restart_noalloc,
 * which restarts tree diffs. */
int b2d_create_list(uint32_t chunk_size, int hash_kind, b2d_dedup** out);
/* ~TreeDeduplicator() -- src/tree_approach.cpp:11 (~ListDeduplicator(), src/list_approach.cpp:11) */
int b2d_destroy(b2d_dedup* d);
/* Run all device work of this handle on `cuda_stream` (a cudaStream_t; NULL = the handle's
 * own stream).  No reference counterpart (Kokkos uses its default execution space). */
int b2d_set_stream(b2d_dedup* d, void* cuda_stream);

/* Tuning knobs (no reference counterpart; output bytes never depend on them):
 *   "leaf_tma"          1 = TMA-staged chunk hashing when the chunk size allows (default), 0 = off
 *   "leaf_stages"       TMA ring depth per CTA, 2..16 (0 = default)
 *   "leaf_ctas_per_sm"  resident hashing CTAs per SM, 1..8 (0 = default 3)
 *   "leaf_unit"         staged segment width 16/32/64/128 bytes, narrower than the default only
 *                       (0 = the largest that divides the chunk; MD5 needs >= 64)
 *   "leaf_wait_polls"   0 = the staged kernel's barrier waits have their normal bound
 *                       (default); n > 0 = they give up after n non-blocking polls, so the
 *                       checkpoint fails with B2D_ERR_TIMEOUT (a test of the give-up path)
 *   "map_max_load_pct" digest-map load limit, 10..90 (default 75): a checkpoint starts only
 *                       when the map's entries plus every node of the tree fit under it
 *   "map_headroom_pct"  size of a baseline's map over that minimum, 100..1000 (default 150);
 *                       more headroom = fewer growths (allocate + rehash) in a long series
 *   "warp_bands"        forest phases whose lowest levels run as warp tasks (7 levels per task
 *                       in phase 1, 9 in phase 2) instead of CTA bands (10 and 12 levels): bit 0
 *                       phase 1, bit 1 phase 2, 0..3 (default 3); trees whose chunk count is not
 *                       a power of two always use CTA bands
 *   "graph"             0 = launch a checkpoint's kernels one by one on the handle's stream
 *                       (default; measured faster), 1 = replay them as one CUDA graph, 2 = graph
 *                       without the phase-timing events (b2d_phase_times then reads 0) */
int b2d_set_param(b2d_dedup* d, const char* name, int64_t value);

/* checkpoint(header_t&, uint8_t* data_ptr, size_t len, HostMirror& diff_h, bool make_baseline)
 * -- src/tree_approach.cpp:1577-1689, minus the device->host copy: the diff stays in device
 * memory owned by the handle (b2d_diff_device / b2d_copy_diff).  advance_id != 0 also does the
 * `current_id += 1` of the other overloads (:1723, :1747, :1775).  `d_data` is a device buffer
 * of `len` bytes; it is only read. */
int b2d_checkpoint_device(b2d_dedup* d, const void* d_data, uint64_t len, int make_baseline, int advance_id,
                          uint64_t* diff_len);
/* Device address and size of the last diff (valid until the next checkpoint on this handle). */
int b2d_diff_device(b2d_dedup* d, const void** d_diff, uint64_t* diff_len);
/* Copy the last diff to host memory `dst` of `cap` bytes (timers[3] of the reference). */
int b2d_copy_diff(b2d_dedup* d, void* dst, uint64_t cap);
/* The same copy enqueued on `cuda_stream` (NULL = the handle's stream) without waiting: `dst`
 * (pinned host memory for an asynchronous copy) holds the diff once that stream reaches this
 * point.  For callers that overlap the copy-back with other checkpoints.  No reference
 * counterpart. */
int b2d_copy_diff_async(b2d_dedup* d, void* dst, uint64_t cap, void* cuda_stream);
/* The three CSV logs of the last checkpoint, as checkpoint(.., logname, ..) writes them
 * (write_chkpt_log, src/tree_approach.cpp:1853-1896 with src/utils.cpp:38-124; "List" rows for
 * a list handle), for a checkpoint taken with b2d_checkpoint_device whose diff is copied back
 * asynchronously: its Write Time column is 0, the copy-back being the caller's.  The checkpoint
 * id written is the diff's.  Reads only the diff's header and repeat table from the device. */
int b2d_write_chkpt_log(b2d_dedup* d, const char* logname);
/* write_chkpt_log(header_t& header, HostMirror& diff_h, std::string& logname)
 * -- include/deduplicator_interface.hpp:172-174, src/tree_approach.cpp:1853-1896 with
 * src/utils.cpp:38-124.  The three CSV logs from a host diff: the 32-byte `header` gives the
 * metadata breakdown's counts, `diff` (diff_len bytes, header first) its repeat table; the
 * Chkpt ID column is the handle's current_id, the Setup/Comparison/Gather/Write times and data
 * sizes the handle's last checkpoint's, as the reference writes them.  B2D_ERR_FORMAT when the
 * diff is shorter than the header's lists. */
int b2d_write_chkpt_log_host(b2d_dedup* d, const void* header, const uint8_t* diff, uint64_t diff_len,
                             const char* logname);
/* write_restart_log(uint32_t select_chkpt, std::string& logname)
 * -- include/deduplicator_interface.hpp:181-182, src/tree_approach.cpp:1904-1915.  Appends one
 * row (approach, select_chkpt, chunk size, the last restart's copy time and total time); a log
 * that cannot be opened is skipped, as in the reference. */
int b2d_write_restart_log(b2d_dedup* d, uint32_t select_chkpt, const char* logname);

/* checkpoint(uint8_t* data_ptr, size_t len, HostMirror& diff_h, bool make_baseline)
 * -- src/tree_approach.cpp:1740-1748.  *diff points at pinned host memory owned by the handle,
 * valid until the next call on it. */
int b2d_checkpoint(b2d_dedup* d, const void* d_data, uint64_t len, int make_baseline, const uint8_t** diff,
                   uint64_t* diff_len);
/* checkpoint(uint8_t* data_ptr, size_t len, HostMirror& diff_h, std::string& logname,
 * bool make_baseline) -- src/tree_approach.cpp:1765-1776 (writes the three CSV logs). */
int b2d_checkpoint_log(b2d_dedup* d, const void* d_data, uint64_t len, const char* logname, int make_baseline,
                       const uint8_t** diff, uint64_t* diff_len);
/* checkpoint(uint8_t* data_ptr, size_t len, std::string& filename, std::string& logname,
 * bool make_baseline) -- src/tree_approach.cpp:1705-1724 (diff written to `filename`).  If the
 * log or the file cannot be written (B2D_ERR_IO) the checkpoint id does not advance and the
 * handle accepts only a baseline next. */
int b2d_checkpoint_file(b2d_dedup* d, const void* d_data, uint64_t len, const char* filename, const char* logname,
                        int make_baseline);

/* restart(uint8_t* data_ptr, size_t len, vector<HostMirror>& chkpts, std::string& logname,
 * uint32_t chkpt_id) -- src/tree_approach.cpp:1807-1813 -> restart_chkpt :712-1128.
 * Rebuilds checkpoint `chkpt_id` into the device buffer `d_out` (len >= the header's datalen;
 * datalen bytes are written, the rest untouched) from host diffs[0..num_diffs).  `logname`
 * may be NULL (no restart log).  diffs[i] must be checkpoint i: a main diff whose header has
 * ref_id > chkpt_id, or a chkpt_id other than `chkpt_id`, is rejected with B2D_ERR_FORMAT before
 * any device work (the reference does not check and rebuilds from the main diff alone). */
int b2d_restart(b2d_dedup* d, void* d_out, uint64_t len, const uint8_t* const* diffs, const uint64_t* sizes,
                uint32_t num_diffs, uint32_t chkpt_id, const char* logname);
/* restart(View data, vector<string>& chkpt_filenames, std::string& logname, uint32_t chkpt_id)
 * -- src/tree_approach.cpp:1827-1838: reads "<name>.hashtree.incr_chkpt" for each name.
 * Offsets are 64-bit (the host-view semantics); the reference's file path computes them in
 * 32 bits (:1265-1290) and breaks above 4 GiB. */
int b2d_restart_files(b2d_dedup* d, void* d_out, uint64_t len, const char* const* chkpt_filenames,
                      uint32_t num_files, uint32_t chkpt_id, const char* logname);

/* b2d_restart with the diffs already in device memory (d_diffs[i]: device pointer, sizes[i]:
 * bytes): no host copies of the diffs, only of their 32-byte headers and repeat tables, so a
 * restart chain kept on the GPU runs at device speed.  No reference counterpart (the
 * reference's restart takes host views, src/tree_approach.cpp:1807-1813). */
int b2d_restart_device(b2d_dedup* d, void* d_out, uint64_t len, const void* const* d_diffs, const uint64_t* sizes,
                       uint32_t num_diffs, uint32_t chkpt_id);

/* Restart that allocates nothing (no counterpart in the reference).  For callers that cannot
 * call cudaMalloc: a process restoring a checkpoint after the device ran out of memory, or a
 * runtime whose device memory is all owned by its own pool and budget.  Same result as
 * b2d_restart, but the diffs are device-resident (d_diffs[i]: device pointer, sizes[i]: bytes)
 * and no handle is needed.  The scratch is one fixed __device__ array in the library (about
 * 10.0 MB on every GPU that loads it, held until exit): at most 2^18 chunks per checkpoint and
 * checkpoint ids below 4096, else B2D_ERR_UNSUPPORTED.  Every call looks up that array's
 * device address for the current device (so it stays right after a cudaDeviceReset); the first
 * call on a device should come before any stream capture.  The same header checks as
 * b2d_restart (B2D_ERR_FORMAT).  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller.  Work runs on
 * `cuda_stream` (NULL = legacy default stream) and the call returns after it completes. */
int b2d_restart_noalloc(void* d_out, uint64_t len, const void* const* d_diffs, const uint64_t* sizes,
                        uint32_t num_diffs, uint32_t chkpt_id, void* cuda_stream);

/* num_first_ocur() / num_shift_dupl() -- include/tree_approach.hpp:53-59 */
int b2d_num_first_ocur(b2d_dedup* d, uint64_t* out);
int b2d_num_shift_dupl(b2d_dedup* d, uint64_t* out);
/* BaseDeduplicator state (include/deduplicator_interface.hpp:16-23) */
int b2d_current_id(b2d_dedup* d, uint32_t* out);
int b2d_baseline_id(b2d_dedup* d, uint32_t* out);
/* timers[4]: setup, comparison (dedup), gather, copy diff to host -- seconds */
int b2d_timers(b2d_dedup* d, double out[4]);
/* restart_timers[2]: copy time, total restart time -- seconds */
int b2d_restart_timers(b2d_dedup* d, double out[2]);
/* datasizes: (data bytes incl. header, metadata bytes) of the last diff (:707-709) */
int b2d_datasizes(b2d_dedup* d, uint64_t out[2]);
/* Device time (seconds, CUDA events on the handle's stream) of the last checkpoint's three
 * stages: chunk hashing + labelling, Merkle forest, diff assembly.  *leaf_path (nullable) is 1
 * when the TMA-staged hashing kernel ran, 0 for the byte-granular one.  No reference
 * counterpart (the reference times whole phases on the host, src/tree_approach.cpp:1640-1688). */
int b2d_phase_times(b2d_dedup* d, double out[3], int* leaf_path);
/* device kernels launched by the last checkpoint/restart call on this handle */
int b2d_last_launch_count(b2d_dedup* d, uint32_t* out);

/* Introspection for tests: copy the first `nodes` tree digests (16 B each, heap order) or the
 * labels of the first `leaves` leaves (1 B each, chunk order; Label values of
 * include/utils.hpp:51-57) of the last checkpoint to host memory. */
int b2d_debug_tree(b2d_dedup* d, void* dst, uint64_t nodes);
int b2d_debug_labels(b2d_dedup* d, void* dst, uint64_t leaves);
/* Digest of each `chunk_size` chunk of a device buffer into d_out (16 B per chunk), the
 * reference's hash() (include/hash_functions.hpp:16-20) as a standalone kernel. */
int b2d_hash_chunks(int hash_kind, const void* d_data, uint64_t len, uint32_t chunk_size, void* d_out,
                    void* cuda_stream);

/* Keep `bytes` of device memory mapped for digest maps on the current device (0 = release
 * it).  Growing a map allocates a larger table; allocating memory the driver has not mapped
 * yet costs tens of ms per GB, which a long-running caller (a checkpoint server with a memory
 * budget) pays once here instead of inside a later checkpoint.  Maps are carved out of this
 * memory while it lasts.  No reference counterpart. */
int b2d_pool_reserve(uint64_t bytes);
/* Device bytes a handle holds now (its tree, map, scratch and diff buffers), and the bytes a
 * handle will hold for checkpoints of a `len`-byte buffer (map_max_load_pct 0 = the default
 * 75), for admission against a memory budget.  No reference counterpart. */
int b2d_memory(b2d_dedup* d, uint64_t* bytes);
/* Digest map statistics: out[0] slots, out[1] entries after the last checkpoint, out[2] times
 * the map has grown (rehashed into a larger table), out[3] host seconds spent growing it,
 * out[4] host seconds spent in the allocation calls of all its tables (baselines included). */
int b2d_map_stats(b2d_dedup* d, double out[5]);
int b2d_estimate_memory(uint64_t len, uint32_t chunk_size, int map_max_load_pct, uint64_t* bytes);

/* ---- Batched checkpoints (no counterpart in the reference, whose checkpoint() takes one
 * buffer at a time: src/tree_approach.cpp:1705).  One call checkpoints `count` buffers, each
 * through its own handle (its own tree, map and checkpoint ids), as one CUDA graph: a single
 * persistent hashing kernel takes tiles of 256 chunks of every buffer from a work queue, then
 * each handle's tree and diff work runs on parallel graph branches.  Per handle the result is
 * exactly what b2d_checkpoint_device(handle, d_data[i], lens[i], make_baseline[i], 1, ..)
 * would give: afterwards b2d_diff_device / b2d_copy_diff / b2d_num_first_ocur read it, and
 * the handle's checkpoint id has advanced.  Handles must be distinct within a call.
 * `make_baseline` may be NULL (no forced baselines); `rcs` (nullable) receives each handle's
 * status.  Every handle's arguments are checked before any handle is touched, so a call
 * rejected by B2D_ERR_ARG / B2D_ERR_LEN_CHANGED / B2D_ERR_UNSUPPORTED leaves every handle as it
 * was (`rcs` names the offending entry).  The graph is rebuilt only when a handle's buffers or
 * sizes change. */
typedef struct b2d_batch b2d_batch;
int b2d_batch_create(b2d_batch** out);
int b2d_batch_destroy(b2d_batch* b);
int b2d_batch_set_stream(b2d_batch* b, void* cuda_stream);
/* Tuning: "leaf_stages" (staging ring depth, 0 = 64 KB ring), "leaf_ctas_per_sm" (0 = 3),
 * "tiles_per_pop" (work-queue granule, tiles of 256 chunks), "streams" (graph branches for the
 * per-handle work when "shared" is 0), "shared" (1 = the shared segmented forest/diff launches,
 * default; 0 = per-handle launches on "streams" branches), "warp_bands" (the fused levels of the
 * first forest band, as the handle parameter of that name, default 3), "map_headroom_pct" (the
 * digest-map load factor: table size over its minimum, default 150; a handle whose table was
 * sized otherwise is resized before its next batch), "autotune" (1: coordinate descent over
 * shared, tiles_per_pop, staging, warp_bands {3, 0} and map_headroom_pct {150, 125}, one setting
 * per incremental batch -- seven batches -- measured by device time, a value kept when it is at
 * least 1 % faster; "tuned" reads 1 once it has
 * settled and the knobs then read the chosen values), "graph" (2 = launch a composition directly
 * the first time and as a captured graph from its second batch on, default; 1 = always a graph;
 * 0 = never), "graph_cache" (instantiated graphs kept, one per batch composition, default 16),
 * "batch_diff" (1 = every handle's diff assembly in 12-13 shared launches after all trees are
 * labelled, default; 0 = per handle in its own branch), "batch_forest" (1 = every handle's
 * Merkle-forest phases in shared launches, one per tree step, default; needs batch_diff).
 * A batch applies its warp_bands and map_headroom_pct to every handle it checkpoints.
 * Output never depends on them. */
int b2d_batch_set_param(b2d_batch* b, const char* name, int64_t value);
int b2d_batch_get_param(b2d_batch* b, const char* name, int64_t* value);
int b2d_batch_checkpoint(b2d_batch* b, b2d_dedup* const* handles, const void* const* d_data, const uint64_t* lens,
                         const int* make_baseline, uint32_t count, int* rcs);
/* The same in two halves, for a caller that keeps several batches in flight (one per batch
 * object, each on its own stream): launch returns once the batch's graph is launched; query
 * sets *done to 1 when its device work has completed (0: running, -1: nothing in flight);
 * wait blocks until then and completes every handle's checkpoint (rcs as above).  A batch
 * object holds one batch at a time, and a handle may be in one batch in flight at a time. */
int b2d_batch_launch(b2d_batch* b, b2d_dedup* const* handles, const void* const* d_data, const uint64_t* lens,
                     const int* make_baseline, uint32_t count, int* rcs);
int b2d_batch_query(b2d_batch* b, int* done);
int b2d_batch_wait(b2d_batch* b, int* rcs);
/* out[0]: device seconds of the last batch (CUDA events around the graph); out[1]: host
 * seconds from the start of its launch to the end of its completion */
int b2d_batch_times(b2d_batch* b, double out[2]);
int b2d_batch_launch_count(b2d_batch* b, uint32_t* out);

/* The same digest of a host buffer, computed on the host (for tools that print the
 * reference's checkpoint digests, include/hash_functions.hpp:47-63).  No device work. */
int b2d_hash_host(int hash_kind, const void* data, uint64_t len, void* out16);

const char* b2d_strerror(int status);

#ifdef __cplusplus
}
#endif

#endif /* B200DEDUP_H */
