// Snapshot history on disk (storage_mode 2): one file per snapshot kind, the
// stored step q at byte offset q * step_bytes (all shots of a step
// contiguous), as the reference's disk mode lays it out
// (storage_utils.cu:36-274, maxwell_tm_cuda_inst.cu:1426-1560).
//
// Writes go through a pinned staging ring (the caller's *_store_3 buffer in
// this mode): the compute side copies a stored step from its device ring slot
// into staging slot q % slots on a CUDA stream, records an event and queues a
// write; one worker thread per file waits for that event and pwrite()s the
// slot.  Before a staging slot is reused its previous write must have
// finished (wait_slot).  Reads (adjoint) are synchronous pread()s into a
// staging slot whose previous host-to-device copy the caller has waited for.
// I/O errors are recorded and reported by finish() / read(); nothing aborts.
#pragma once

#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <cerrno>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace tb {

class DiskHistory {
 public:
  // Opens path for writing (write = true; the file is created if missing and
  // not truncated, so a history written over several calls keeps its earlier
  // steps) or reading.
  DiskHistory(const char *path, bool write, int slots)
      : busy_(static_cast<size_t>(slots), 0), write_(write) {
    fd_ = ::open(path, write ? (O_CREAT | O_WRONLY) : O_RDONLY, 0600);
    if (fd_ < 0) {
      error_ = std::string("open(") + path + ") failed: " + std::strerror(errno);
      return;
    }
    if (write) worker_ = std::thread(&DiskHistory::run, this);
  }
  ~DiskHistory() { finish(); }
  DiskHistory(const DiskHistory &) = delete;
  DiskHistory &operator=(const DiskHistory &) = delete;

  bool ok() const { return fd_ >= 0 && error_.empty(); }
  const std::string &error() const { return error_; }

  // Blocks until the staging slot's queued write (if any) has completed.
  void wait_slot(int slot) {
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return busy_[static_cast<size_t>(slot)] == 0; });
  }

  // Queues: once `ready` has completed, write nbytes from src at offset.
  void enqueue_write(int slot, const void *src, size_t nbytes, int64_t offset,
                     cudaEvent_t ready) {
    std::lock_guard<std::mutex> lk(mu_);
    busy_[static_cast<size_t>(slot)] = 1;
    q_.push_back(Task{slot, src, nbytes, offset, ready});
    cv_task_.notify_one();
  }

  // Synchronous read of nbytes at offset into dst.
  bool read(void *dst, size_t nbytes, int64_t offset) {
    char *p = static_cast<char *>(dst);
    size_t done = 0;
    while (done < nbytes) {
      const ssize_t k = ::pread(fd_, p + done, nbytes - done, (off_t)(offset + (int64_t)done));
      if (k <= 0) {
        if (k < 0 && errno == EINTR) continue;
        error_ = k == 0 ? "pread: unexpected end of snapshot file"
                        : std::string("pread failed: ") + std::strerror(errno);
        return false;
      }
      done += (size_t)k;
    }
    return true;
  }

  // Waits for every queued write, stops the worker and closes the file.
  bool finish() {
    if (worker_.joinable()) {
      {
        std::lock_guard<std::mutex> lk(mu_);
        closing_ = true;
        cv_task_.notify_all();
      }
      worker_.join();
    }
    if (fd_ >= 0) {
      if (write_ && ::fsync(fd_) != 0 && error_.empty())
        error_ = std::string("fsync failed: ") + std::strerror(errno);
      ::close(fd_);
      fd_ = -1;
    }
    return error_.empty();
  }

 private:
  struct Task {
    int slot;
    const void *src;
    size_t nbytes;
    int64_t offset;
    cudaEvent_t ready;
  };

  void run() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_task_.wait(lk, [&] { return closing_ || !q_.empty(); });
        if (q_.empty()) return;  // closing and drained
        t = q_.front();
        q_.pop_front();
      }
      std::string err;
      if (cudaEventSynchronize(t.ready) != cudaSuccess) {
        cudaGetLastError();
        err = "staging copy to host failed";
      }
      const char *p = static_cast<const char *>(t.src);
      size_t done = 0;
      while (err.empty() && done < t.nbytes) {
        const ssize_t k =
            ::pwrite(fd_, p + done, t.nbytes - done, (off_t)(t.offset + (int64_t)done));
        if (k < 0 && errno == EINTR) continue;
        if (k <= 0) {
          err = std::string("pwrite failed: ") + std::strerror(errno);
          break;
        }
        done += (size_t)k;
      }
      std::lock_guard<std::mutex> lk(mu_);
      if (!err.empty() && error_.empty()) error_ = err;
      busy_[static_cast<size_t>(t.slot)] = 0;
      cv_done_.notify_all();
    }
  }

  int fd_ = -1;
  std::vector<char> busy_;
  bool write_;
  bool closing_ = false;
  std::deque<Task> q_;
  std::mutex mu_;
  std::condition_variable cv_task_, cv_done_;
  std::string error_;
  std::thread worker_;
};

}  // namespace tb
