// Declarations shared by every translation unit of the dfjk library: constants,
// errors, device buffers and shell tables. Kept apart from internal.h (plans,
// contexts) so that the integral kernels do not recompile when those change.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <cstdint>
#include <cstdio>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dfjk.h"

namespace dfjk {

// Count of this library's kernel launches (host-side, all contexts).
void count_launch(int64_t n = 1);

// Angular-momentum coverage of the compiled integral kernels.
constexpr int kLmaxOrb = 3;   // orbital shells up to f
constexpr int kLmaxAux = 4;   // auxiliary shells up to g

// Boys table geometry (dftax/energy/boys.py:33-36).
constexpr int kBoysOrder = 6;
constexpr int kBoysNmax = 24;
constexpr int kBoysNgrid = 401;
constexpr double kBoysDt = 0.1;
constexpr double kBoysTmax = 40.0;

struct Error {
  dfjk_status code;
  std::string msg;
};

[[noreturn]] void fail(dfjk_status code, const char* fmt, ...);

#define DFJK_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      ::dfjk::fail(DFJK_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                   __FILE__, __LINE__);                                              \
  } while (0)

#define DFJK_CUBLAS(call)                                                            \
  do {                                                                               \
    cublasStatus_t s_ = (call);                                                      \
    if (s_ != CUBLAS_STATUS_SUCCESS)                                                 \
      ::dfjk::fail(DFJK_ERR_CUDA, "%s failed: cublas status %d (%s:%d)", #call, (int)s_, \
                   __FILE__, __LINE__);                                              \
  } while (0)

#define DFJK_CUSOLVER(call)                                                          \
  do {                                                                               \
    cusolverStatus_t s_ = (call);                                                    \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                               \
      ::dfjk::fail(DFJK_ERR_CUDA, "%s failed: cusolver status %d (%s:%d)", #call, (int)s_, \
                   __FILE__, __LINE__);                                              \
  } while (0)

// After every kernel launch: surface launch errors and count the launch.
#define DFJK_LAUNCHED()                 \
  do {                                  \
    DFJK_CUDA(cudaGetLastError());      \
    ::dfjk::count_launch();             \
  } while (0)

// Device memory cache (api.cu): freed DevBufs are kept for reuse per device.
// Synchronizes device dev and records that every buffer freed before the
// synchronization began is idle (may be handed out again without waiting).
void sync_device(int dev);
void cache_trim(int dev);            // cudaFree every cached buffer of dev
// Held while a stream of this library captures a CUDA graph, and by every
// device-wide synchronization (cudaDeviceSynchronize, cudaFree) the library
// makes: those fail while any stream of the device is capturing, and the
// batch engine's workers capture and allocate from different threads.
std::recursive_mutex& capture_mutex();

// Runs fn(t) for t = 0 .. T-1: t > 0 on host threads, t = 0 on the caller. A
// thread that cannot be started runs on the caller instead; the first
// exception any call throws is rethrown once every thread has joined.
template <class F>
void run_on_threads(int T, F&& fn) {
  std::exception_ptr err;
  std::mutex mu;
  auto call = [&](int t) {
    try {
      fn(t);
    } catch (...) {
      std::lock_guard<std::mutex> lk(mu);
      if (!err) err = std::current_exception();
    }
  };
  std::vector<std::thread> th;
  int started = 1;
  try {
    th.reserve(T > 1 ? T - 1 : 0);
    for (; started < T; ++started) th.emplace_back(call, started);
  } catch (...) {
  }
  for (int t = started; t < T; ++t) call(t);
  call(0);
  for (auto& x : th) x.join();
  if (err) std::rethrow_exception(err);
}

// Device buffer owned by a plan or context (allocated through the cache).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int dev = 0;
  void alloc(size_t n);
  void free();
  // grow-only: keep the allocation when it is already large enough
  void ensure(size_t n) {
    if (!p || bytes < n) alloc(n);
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
  ~DevBuf() { free(); }
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

template <class T>
void upload(DevBuf& b, const std::vector<T>& v) {
  b.alloc(v.size() * sizeof(T) + 16);
  if (!v.empty()) DFJK_CUDA(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}

// Shell table of one basis (host side and device mirror).
struct Shells {
  int n = 0;
  std::vector<int> l, nprim, prim0, row0, out0, ncomp;
  std::vector<double> cen;            // 3 per shell
  std::vector<double> pexp, pcoef;    // per primitive
  int ncart = 0, nout = 0, lmax = 0;
  bool spherical = true;
  // device
  DevBuf d_l, d_nprim, d_prim0, d_cen, d_pexp, d_pcoef;
  void reset() {
    n = ncart = nout = lmax = 0;
    spherical = true;
    l.clear(); nprim.clear(); prim0.clear(); row0.clear(); out0.clear(); ncomp.clear();
    cen.clear(); pexp.clear(); pcoef.clear();
  }
};

// Transformation blocks, one per l: ncart(l) x nout(l), row-major, packed.
struct Blocks {
  std::vector<double> host;
  int off[8] = {0};
  DevBuf dev;
  void reset() {
    host.clear();
    for (int& o : off) o = 0;
  }
};

// Device-side views passed to kernels.
struct ShellView {
  const int* l;
  const int* nprim;
  const int* prim0;
  const double* cen;
  const double* pexp;
  const double* pcoef;
};

}  // namespace dfjk
