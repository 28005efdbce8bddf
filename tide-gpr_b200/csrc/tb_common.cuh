// Host-side status reporting shared by every entry point of libtide_b200.so.
//
// The reference reports CUDA errors with fprintf and then calls std::exit or
// abort (src/tide/csrc/common/common_gpu.h:12-31).  Here no entry point ever
// terminates the process: a failure is recorded as (status, message) and the
// call returns early; callers read it through tide_b200_last_status() /
// tide_b200_last_error().
#pragma once

#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdint>
#include <cstdio>

namespace tb {

enum Status : int {
  kOk = 0,
  kBadArgument = 1,
  kCudaError = 2,
  kNotBuilt = 3,
};

void set_error(int status, const char *fmt, ...);

// Record a CUDA failure; returns true when `e` is an error.
bool cuda_failed(cudaError_t e, const char *what, const char *file, int line);

// Launch accounting and optional per-kernel event timing (benchmarks).
enum KernelKind : int {
  kKFwdH = 0,     // forward H half step
  kKFwdE = 1,     // forward E half step (+ snapshots, points)
  kKAdjE = 2,     // adjoint E-phase
  kKAdjH = 3,     // adjoint H-phase (+ points, gradient)
  kKFwdStep = 4,  // fused forward step (stencil 2)
  kKAdjStep = 5,  // fused adjoint step (stencil 2)
  kK3FwdH = 6,    // 3-D forward H half step
  kK3FwdE = 7,    // 3-D forward E half step (+ snapshots)
  kK3AdjE = 8,    // 3-D adjoint E-phase
  kK3AdjH = 9,    // 3-D adjoint H-phase
  kK3Grad = 10,   // 3-D coefficient gradient of an imaged step
  kKindCount = 11
};
void count_launches(int64_t n);

// cudaMallocAsync on the current device's default pool, with the pool told
// (once per device) to keep up to 4 GiB of freed memory instead of releasing
// it at every synchronisation, so per-call scratch is a pool hit after the
// first call while larger transient use still goes back to the driver.
cudaError_t pool_malloc(void **p, size_t bytes, cudaStream_t st);

// Brackets sampled launches with events on one stream; accumulates into the
// process-wide profile when the scope closes (after waiting for its events).
//
// Launches captured into a CUDA graph are timed by event-record nodes: between
// capture_begin and capture_end, begin / end add such nodes on the capture
// stream (their events are placeholders); bind maps them to the instantiated
// graph's nodes, and arm gives those nodes fresh events before each timed
// replay, so every replay's times are kept.
class ProfileScope {
 public:
  explicit ProfileScope(cudaStream_t st);
  ~ProfileScope();
  bool on() const { return on_; }
  bool sample(int64_t step) const;  // is this time step timed?
  void begin(int kind);
  void end(int kind);
  void capture_begin(cudaStream_t cs);
  void capture_end();
  bool bind(cudaGraph_t graph);        // false: no timed nodes (or an error)
  bool arm(cudaGraphExec_t exec);      // before each timed replay of `exec`

 private:
  cudaStream_t st_;
  bool on_;
  int every_;
  int open_kind_ = -1;
  struct Pair { cudaEvent_t a, b; int kind; };
  Pair *pairs_ = nullptr;
  int n_ = 0, cap_ = 0;
  bool push(cudaEvent_t a, cudaEvent_t b, int kind);
  // graph timing: placeholder pairs recorded during capture and their nodes
  cudaStream_t cs_ = nullptr;
  struct NodePair { cudaEvent_t a, b; cudaGraphNode_t na, nb; int kind; };
  NodePair *tmpl_ = nullptr;
  int nt_ = 0, tcap_ = 0;
};

}  // namespace tb

#define TB_CUDA(call)                                                         \
  (tb::cuda_failed((call), #call, __FILE__, __LINE__))

#define TB_REQUIRE(cond, ...)                                                 \
  do {                                                                        \
    if (!(cond)) {                                                            \
      tb::set_error(tb::kBadArgument, __VA_ARGS__);                           \
      return;                                                                 \
    }                                                                         \
  } while (0)

// TB_REQUIRE for helpers that report failure by returning false.
#define TB_REQUIRE_B(cond, ...)                                               \
  do {                                                                        \
    if (!(cond)) {                                                            \
      tb::set_error(tb::kBadArgument, __VA_ARGS__);                           \
      return false;                                                           \
    }                                                                         \
  } while (0)
