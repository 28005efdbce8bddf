// Snapshot history of a storing forward pass, shared by the TM2D, Born and
// 3-D storing forwards (maxwell_tm_cuda_inst.cu:1281-1609 and 1701-2086 and
// maxwell_3d_cuda_inst.cu:3290-3880 run the same pipeline).  K snapshot kinds
// (2-D: Ey and curl H; 3-D: three E and three curl H components), each with a
// device buffer s1, a host buffer s3 and a file-name list fn.
//
// Storage modes: 0 device (the whole history in s1), 1 cpu (3-slot device
// ring in s1, pinned host history in s3), 2 disk (device ring, 3-slot pinned
// staging ring in s3, one file per kind written by a DiskHistory thread),
// 3 none.  Store index q = t / step_ratio sits at q * step_bytes of its
// history (device, host or file).  With a storage stream distinct from the
// compute stream, the device-to-host copies run on it and overlap the next
// steps' kernels; events keep a ring slot from being overwritten before its
// copy ran.
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "tb_common.cuh"
#include "tb_disk.cuh"

namespace tb {
namespace {

constexpr int kStoreRing = 3;  // device ring slots (NUM_BUFFERS, maxwell.cu:45-47)

struct EventRing {
  cudaEvent_t ev[kStoreRing]{};
  bool ok = true;
  EventRing() {
    for (auto &e : ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) ok = false;
  }
  ~EventRing() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
};

template <int K>
struct StoreRun {
  const char *who = "";
  bool want = false, bf16 = false, host_side = false, pipeline = false, to_disk = false;
  int64_t mode = 3, step_ratio = 1;
  size_t step_bytes = 0;
  char *s1[K] = {}, *s3[K] = {};
  cudaStream_t st = nullptr, ss = nullptr;
  std::unique_ptr<DiskHistory> disk[K];
  EventRing staged;                    // a staging slot's device-to-host copy is done
  EventRing store_done, compute_done;  // cpu/disk pipeline on the storage stream

  // Validates the storage arguments; false (with the error set) on bad ones.
  // need[k]: kind k is stored; cells: elements of one shot of one kind.
  bool init(const char *name, const bool need[K], int64_t storage_mode, int64_t storage_format,
            size_t field_size, int64_t shot_bytes_uncomp, int64_t cells, int64_t n_shots,
            int64_t ratio, void *const dev[K], void *const host[K],
            char const *const *const files[K], cudaStream_t compute, cudaStream_t storage) {
    who = name;
    TB_REQUIRE_B(storage_mode >= 0 && storage_mode <= 3, "%s: unknown storage_mode %lld", who,
                 (long long)storage_mode);
    bf16 = storage_format == 1;
    TB_REQUIRE_B(!bf16 || field_size == 4, "%s: bf16 snapshot storage requires float32 fields",
                 who);
    bool any = false;
    for (int k = 0; k < K; ++k) any = any || need[k];
    want = any && storage_mode != 3;
    mode = storage_mode;
    step_ratio = ratio;
    st = compute;
    ss = storage;
    if (!want) return true;
    const size_t esz = bf16 ? 2 : field_size;
    TB_REQUIRE_B(shot_bytes_uncomp == cells * (int64_t)esz,
                 "%s: shot_bytes_uncomp=%lld does not match cells*elem=%lld", who,
                 (long long)shot_bytes_uncomp, (long long)(cells * (int64_t)esz));
    host_side = mode == 1 || mode == 2;
    to_disk = mode == 2;
    for (int k = 0; k < K; ++k) {
      if (!need[k]) continue;
      TB_REQUIRE_B(dev[k], "%s: snapshot buffers missing", who);
      TB_REQUIRE_B(!host_side || host[k], "%s: cpu / disk storage modes need host snapshot buffers",
                   who);
      TB_REQUIRE_B(!to_disk || (files[k] && files[k][0]),
                   "%s: disk storage mode needs snapshot file names", who);
      s1[k] = (char *)dev[k];
      s3[k] = (char *)host[k];
    }
    step_bytes = (size_t)shot_bytes_uncomp * (size_t)n_shots;
    pipeline = host_side && ss != nullptr && ss != st;
    if (to_disk) {
      if (!staged.ok) {
        set_error(kCudaError, "%s: event creation failed", who);
        return false;
      }
      for (int k = 0; k < K; ++k)
        if (s1[k]) {
          disk[k].reset(new DiskHistory(files[k][0], true, kStoreRing));
          if (!disk[k]->ok()) {
            set_error(kBadArgument, "%s disk storage: %s", who, disk[k]->error().c_str());
            return false;
          }
        }
    }
    if (pipeline) {
      if (!store_done.ok || !compute_done.ok) {
        set_error(kCudaError, "%s: event creation failed", who);
        return false;
      }
      for (int k = 0; k < kStoreRing; ++k)
        if (TB_CUDA(cudaEventRecord(store_done.ev[k], ss))) return false;
    }
    return true;
  }

  bool stores(int64_t t) const { return want && (t % step_ratio) == 0; }

  // Device slots that step t writes (null when the step stores nothing); the
  // compute stream waits until the slot's previous host copy has run.
  bool begin(int64_t t, char *dst[K]) {
    for (int k = 0; k < K; ++k) dst[k] = nullptr;
    if (!stores(t)) return true;
    const int64_t q = t / step_ratio;
    const int slot = (int)(q % kStoreRing);
    const size_t off = mode == 0 ? (size_t)q * step_bytes : (size_t)slot * step_bytes;
    for (int k = 0; k < K; ++k)
      if (s1[k]) dst[k] = s1[k] + off;
    return !(pipeline && TB_CUDA(cudaStreamWaitEvent(st, store_done.ev[slot], 0)));
  }

  // After step t's launches: cpu mode copies the slots into the host history;
  // disk mode copies them into the staging slot (whose previous write must
  // have finished) and queues the slot for the file.
  bool end(int64_t t, char *const dst[K]) {
    if (!stores(t) || !host_side) return true;
    const int64_t q = t / step_ratio;
    const int slot = (int)(q % kStoreRing);
    cudaStream_t cs = st;
    if (pipeline) {
      if (TB_CUDA(cudaEventRecord(compute_done.ev[slot], st))) return false;
      if (TB_CUDA(cudaStreamWaitEvent(ss, compute_done.ev[slot], 0))) return false;
      cs = ss;
    }
    const size_t off3 = to_disk ? (size_t)slot * step_bytes : (size_t)q * step_bytes;
    for (int k = 0; k < K; ++k) {
      if (!dst[k]) continue;
      if (to_disk) disk[k]->wait_slot(slot);
      if (TB_CUDA(cudaMemcpyAsync(s3[k] + off3, dst[k], step_bytes, cudaMemcpyDeviceToHost, cs)))
        return false;
    }
    if (to_disk) {
      if (TB_CUDA(cudaEventRecord(staged.ev[slot], cs))) return false;
      for (int k = 0; k < K; ++k)
        if (dst[k])
          disk[k]->enqueue_write(slot, s3[k] + off3, step_bytes, (int64_t)(q * step_bytes),
                                 staged.ev[slot]);
    }
    return !(pipeline && TB_CUDA(cudaEventRecord(store_done.ev[slot], ss)));
  }

  // The call returns once the host history is complete and the files written.
  bool finish() {
    if (host_side && TB_CUDA(cudaStreamSynchronize(pipeline ? ss : st))) return false;
    for (int k = 0; k < K; ++k)
      if (disk[k] && !disk[k]->finish()) {
        set_error(kCudaError, "%s disk storage: %s", who, disk[k]->error().c_str());
        return false;
      }
    return true;
  }
};

}  // namespace
}  // namespace tb
