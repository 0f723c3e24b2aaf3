// Host-side engine behind the C ABI: device memory, per-axis tables, the
// CUDA-graph-captured step, FP64 reductions and checkpoints.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/quasi_gpu.h"
#include "step_impl.cuh"

namespace quasi {

class EngineBase {
 public:
  virtual ~EngineBase() {}
  virtual int set_psi(const double* host) = 0;
  virtual int init() = 0;
  virtual int step(int nsteps, double* device_ms) = 0;
  virtual int step_async(int nsteps) = 0;
  virtual int synchronize() = 0;
  virtual int get_field(int field, double* host) = 0;
  virtual int diagnostics(double out[3]) = 0;
  virtual int growth_rate(double* out) = 0;
  virtual int save(const char* path) = 0;
  virtual int load(const char* path) = 0;
  virtual long nloop() const = 0;
  virtual int step_kernels(int* n) = 0;
  virtual int time_axis_pass(int axis, int reps, double* avg_ms) = 0;
  // The captured step graph of rotation phase `ph` (owned by the engine), for
  // an ensemble that launches all its members' steps as one graph; nullptr
  // before the graphs exist.
  virtual cudaGraph_t phase_graph(int ph) const = 0;
  virtual int phases() const = 0;
  virtual int device() const = 0;
  // steps launched for this engine by such a graph (host counter only)
  virtual void note_steps(int n) = 0;
  virtual bool initialized() const = 0;
  virtual void tuning(int out[4]) const = 0;
  std::string err;
};

EngineBase* make_engine_f64(const quasi_config& cfg, std::string& err);
EngineBase* make_engine_f32(const quasi_config& cfg, std::string& err);

// Host loop over [0, n) split into contiguous chunks on up to 16 threads (the
// field conversions between the caller's doubles and the staging buffer).
template <class F>
inline void host_parallel(size_t n, F&& f) {
  unsigned hw = std::thread::hardware_concurrency();
  const size_t nt = std::min<size_t>(hw ? hw : 1, 16);
  if (nt <= 1 || n < (size_t(1) << 20)) {
    f(size_t(0), n);
    return;
  }
  std::vector<std::thread> pool;
  const size_t chunk = (n + nt - 1) / nt;
  for (size_t t = 1; t < nt; ++t) {
    const size_t lo = std::min(n, t * chunk), hi = std::min(n, lo + chunk);
    pool.emplace_back([&f, lo, hi] { f(lo, hi); });
  }
  f(size_t(0), std::min(n, chunk));
  for (auto& th : pool) th.join();
}

// Validates a configuration; returns an empty string when it is usable.
std::string validate_config(const quasi_config& c);

// exp(-2 pi i t / n), exp(-i pi k / 2n) in long double, rounded to T
template <typename T>
void make_twiddles(int n, std::vector<Cx<T>>& root, std::vector<Cx<T>>& quarter) {
  const long double pi = 3.14159265358979323846264338327950288L;
  root.resize(n);
  quarter.resize(n);
  for (int t = 0; t < n; ++t) {
    long double a = -2.0L * pi * t / n;
    root[t] = Cx<T>{T(std::cos(a)), T(std::sin(a))};
    long double b = -pi * t / (2.0L * n);
    quarter[t] = Cx<T>{T(std::cos(b)), T(std::sin(b))};
  }
}

// Device copy of one axis's twiddles.
template <typename T>
struct DevTwiddles {
  Cx<T>* root = nullptr;
  Cx<T>* quarter = nullptr;
  cudaError_t upload(int n) {
    std::vector<Cx<T>> r, q;
    make_twiddles<T>(n, r, q);
    cudaError_t e;
    if ((e = cudaMalloc(&root, n * sizeof(Cx<T>))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&quarter, n * sizeof(Cx<T>))) != cudaSuccess) return e;
    if ((e = cudaMemcpy(root, r.data(), n * sizeof(Cx<T>), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    return cudaMemcpy(quarter, q.data(), n * sizeof(Cx<T>), cudaMemcpyHostToDevice);
  }
  void release() {
    if (root) cudaFree(root);
    if (quarter) cudaFree(quarter);
    root = quarter = nullptr;
  }
  Tables<T> tables() const { return Tables<T>{root, quarter}; }
};

}  // namespace quasi
