// Process-wide status record and the small metadata entry points.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <vector>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/tide_b200.h"
#include "tb_common.cuh"
#include "tb_tma.cuh"

#include <cudaTypedefs.h>

namespace tb {

namespace {
std::mutex g_mu;
std::atomic<int> g_status{0};
std::string g_message;
}  // namespace

void set_error(int status, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  std::lock_guard<std::mutex> lk(g_mu);
  g_status.store(status);
  g_message = buf;
}

bool cuda_failed(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return false;
  set_error(kCudaError, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  return true;
}

namespace {
std::atomic<int64_t> g_launches{0};
std::atomic<int> g_prof_on{0};
std::atomic<int> g_prof_every{8};
std::mutex g_prof_mu;
double g_prof_ms[kKindCount] = {};
int64_t g_prof_n[kKindCount] = {};
// Event pool shared by all scopes (events are reused across calls).
std::mutex g_pool_mu;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take_event() {
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool.empty()) {
      cudaEvent_t e = g_pool.back();
      g_pool.pop_back();
      return e;
    }
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}
void give_event(cudaEvent_t e) {
  if (!e) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  g_pool.push_back(e);
}
}  // namespace

void count_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

cudaError_t pool_malloc(void **p, size_t bytes, cudaStream_t st) {
  static std::atomic<uint64_t> kept{0};  // bit d: device d's pool configured
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 64 && !(kept.load() & (1ull << dev))) {
    cudaMemPool_t pool;
    uint64_t keep = (uint64_t)4 << 30;  // up to 4 GiB stays mapped between calls
    e = cudaDeviceGetDefaultMemPool(&pool, dev);
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    kept.fetch_or(1ull << dev);
  }
  e = cudaMallocAsync(p, bytes, st);
  if (e == cudaErrorMemoryAllocation) {
    // memory the pool keeps from earlier calls may be what is missing: wait
    // for the stream's pending frees, return the pool's unused memory to the
    // driver and try once more
    cudaGetLastError();
    cudaMemPool_t pool;
    if (cudaStreamSynchronize(st) == cudaSuccess &&
        cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
        cudaMemPoolTrimTo(pool, 0) == cudaSuccess)
      e = cudaMallocAsync(p, bytes, st);
  }
  return e;
}

ProfileScope::ProfileScope(cudaStream_t st)
    : st_(st), on_(g_prof_on.load() != 0), every_(std::max(1, g_prof_every.load())) {}

bool ProfileScope::sample(int64_t step) const { return on_ && (step % every_) == 0; }

bool ProfileScope::push(cudaEvent_t a, cudaEvent_t b, int kind) {
  if (n_ == cap_) {
    int nc = cap_ ? 2 * cap_ : 256;
    Pair *np = static_cast<Pair *>(realloc(pairs_, sizeof(Pair) * nc));
    if (!np) return false;
    pairs_ = np;
    cap_ = nc;
  }
  pairs_[n_++] = Pair{a, b, kind};
  return true;
}

void ProfileScope::begin(int kind) {
  if (!on_) return;
  cudaEvent_t a = take_event(), b = take_event();
  if (!a || !b) {
    give_event(a);
    give_event(b);
    return;
  }
  if (cs_) {  // an event-record node of the graph being captured
    if (nt_ == tcap_) {
      int nc = tcap_ ? 2 * tcap_ : 16;
      NodePair *np = static_cast<NodePair *>(realloc(tmpl_, sizeof(NodePair) * nc));
      if (!np) {
        give_event(a);
        give_event(b);
        return;
      }
      tmpl_ = np;
      tcap_ = nc;
    }
    tmpl_[nt_] = NodePair{a, b, nullptr, nullptr, kind};
    cudaEventRecordWithFlags(a, cs_, cudaEventRecordExternal);
  } else {
    if (!push(a, b, kind)) {
      give_event(a);
      give_event(b);
      return;
    }
    --n_;  // completed by end()
    cudaEventRecord(a, st_);
  }
  open_kind_ = kind;
}

void ProfileScope::end(int kind) {
  if (!on_ || open_kind_ != kind) return;
  if (cs_) {
    cudaEventRecordWithFlags(tmpl_[nt_].b, cs_, cudaEventRecordExternal);
    ++nt_;
  } else {
    cudaEventRecord(pairs_[n_].b, st_);
    ++n_;
  }
  open_kind_ = -1;
}

void ProfileScope::capture_begin(cudaStream_t cs) {
  if (!on_) return;
  cs_ = cs;
  open_kind_ = -1;
}

void ProfileScope::capture_end() { cs_ = nullptr; }

bool ProfileScope::bind(cudaGraph_t graph) {
  if (!on_ || nt_ == 0) return false;
  size_t n = 0;
  if (cudaGraphGetNodes(graph, nullptr, &n) != cudaSuccess) return false;
  std::vector<cudaGraphNode_t> nodes(n);
  if (n == 0 || cudaGraphGetNodes(graph, nodes.data(), &n) != cudaSuccess) return false;
  for (cudaGraphNode_t node : nodes) {
    cudaGraphNodeType type;
    cudaEvent_t ev = nullptr;
    if (cudaGraphNodeGetType(node, &type) != cudaSuccess) return false;
    if (type != cudaGraphNodeTypeEventRecord) continue;
    if (cudaGraphEventRecordNodeGetEvent(node, &ev) != cudaSuccess) return false;
    for (int i = 0; i < nt_; ++i) {
      if (tmpl_[i].a == ev) tmpl_[i].na = node;
      if (tmpl_[i].b == ev) tmpl_[i].nb = node;
    }
  }
  for (int i = 0; i < nt_; ++i)
    if (!tmpl_[i].na || !tmpl_[i].nb) return false;
  return true;
}

bool ProfileScope::arm(cudaGraphExec_t exec) {
  for (int i = 0; i < nt_; ++i) {
    cudaEvent_t a = take_event(), b = take_event();
    if (!a || !b || cudaGraphExecEventRecordNodeSetEvent(exec, tmpl_[i].na, a) != cudaSuccess ||
        cudaGraphExecEventRecordNodeSetEvent(exec, tmpl_[i].nb, b) != cudaSuccess ||
        !push(a, b, tmpl_[i].kind)) {
      give_event(a);
      give_event(b);
      return false;
    }
  }
  return true;
}

// Event pairs of closed scopes wait here until tide_b200_profile_read, so a
// profiled call never blocks the host.
std::mutex g_pending_mu;
std::vector<std::pair<std::pair<cudaEvent_t, cudaEvent_t>, int>> g_pending;

ProfileScope::~ProfileScope() {
  for (int i = 0; i < nt_; ++i) {  // placeholders: recorded by no replay
    give_event(tmpl_[i].a);
    give_event(tmpl_[i].b);
  }
  free(tmpl_);
  if (!on_) return;
  {
    std::lock_guard<std::mutex> lk(g_pending_mu);
    for (int i = 0; i < n_; ++i) g_pending.push_back({{pairs_[i].a, pairs_[i].b}, pairs_[i].kind});
  }
  free(pairs_);
}

void resolve_pending() {
  std::vector<std::pair<std::pair<cudaEvent_t, cudaEvent_t>, int>> pend;
  {
    std::lock_guard<std::mutex> lk(g_pending_mu);
    pend.swap(g_pending);
  }
  double ms[kKindCount] = {};
  int64_t cnt[kKindCount] = {};
  for (auto &p : pend) {
    float t = 0.f;
    if (cudaEventSynchronize(p.first.second) == cudaSuccess &&
        cudaEventElapsedTime(&t, p.first.first, p.first.second) == cudaSuccess) {
      ms[p.second] += t;
      cnt[p.second] += 1;
    }
    give_event(p.first.first);
    give_event(p.first.second);
  }
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (int k = 0; k < kKindCount; ++k) {
    g_prof_ms[k] += ms[k];
    g_prof_n[k] += cnt[k];
  }
}

// Driver entry point of the tensor-map encoder, looked up once through the
// runtime (no link-time dependence on libcuda).
namespace {
PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}
}  // namespace

bool encode_map_3d(CUtensorMap *map, const float *base, int64_t nx, int64_t ny, int64_t nz,
                   int64_t pitch, int bx, int by) {
  auto fn = encoder();
  if (!fn) {
    set_error(kCudaError, "cuTensorMapEncodeTiled is not available from the driver");
    return false;
  }
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)(pitch * ny) * 4};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error(kCudaError,
              "cuTensorMapEncodeTiled failed (%d): dims %lld x %lld x %lld, pitch %lld, box %d x %d",
              (int)r, (long long)nx, (long long)ny, (long long)nz, (long long)pitch, bx, by);
    return false;
  }
  return true;
}

}  // namespace tb

extern "C" {

void tide_b200_profile_enable(int on, int sample_every) {
  tb::g_prof_every.store(sample_every > 0 ? sample_every : 1);
  tb::g_prof_on.store(on ? 1 : 0);
}

int tide_b200_profile_read(double *ms_out, int64_t *launches_out, int max_kinds) {
  tb::resolve_pending();
  std::lock_guard<std::mutex> lk(tb::g_prof_mu);
  int n = max_kinds < tb::kKindCount ? max_kinds : tb::kKindCount;
  for (int k = 0; k < n; ++k) {
    if (ms_out) ms_out[k] = tb::g_prof_ms[k];
    if (launches_out) launches_out[k] = tb::g_prof_n[k];
  }
  for (int k = 0; k < tb::kKindCount; ++k) {
    tb::g_prof_ms[k] = 0.0;
    tb::g_prof_n[k] = 0;
  }
  return tb::kKindCount;
}

const char *tide_b200_profile_kind_name(int kind) {
  static const char *names[] = {"fwd_h",      "fwd_e",      "adj_e",      "adj_h",
                                "fwd_step",   "adj_step",   "em3d_fwd_h", "em3d_fwd_e",
                                "em3d_adj_e", "em3d_adj_h", "em3d_grad"};
  return (kind >= 0 && kind < tb::kKindCount) ? names[kind] : "";
}

int64_t tide_b200_launch_count(void) { return tb::g_launches.load(); }

int tide_b200_release_scratch(int64_t device) {
  cudaMemPool_t pool;
  if (TB_CUDA(cudaSetDevice((int)device)) || TB_CUDA(cudaDeviceSynchronize()) ||
      TB_CUDA(cudaDeviceGetDefaultMemPool(&pool, (int)device)) ||
      TB_CUDA(cudaMemPoolTrimTo(pool, 0)))
    return -1;
  return 0;
}


const char *tide_cuda_arches(void) { return "100a"; }

int tide_b200_last_status(void) { return tb::g_status.load(); }

const char *tide_b200_last_error(void) {
  static thread_local std::string copy;
  std::lock_guard<std::mutex> lk(tb::g_mu);
  copy = tb::g_message;
  return copy.c_str();
}

void tide_b200_clear_error(void) {
  std::lock_guard<std::mutex> lk(tb::g_mu);
  tb::g_status.store(0);
  tb::g_message.clear();
}

}  // extern "C"
