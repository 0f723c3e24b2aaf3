// quasi_r2r_*: one in-place 3-D r2r transform with FFTW's kind semantics,
// the counterpart of fftw_mpi_plan_r2r_3d + fftw_execute (quasi.cpp:449-495).
#include <cuda_runtime.h>

#include <new>
#include <string>
#include <vector>

#include "engine.cuh"

namespace quasi {

struct R2RBase {
  virtual ~R2RBase() {}
  virtual cudaError_t exec(void* data, cudaStream_t s) = 0;
  int nx, ny, nz, device, elem;
  cudaStream_t own = nullptr;
  int* tma_err = nullptr;
  int sms = 148;
  int inject_skip = -1;             // fault injection for the next execution
  uint32_t inject_polls = kTmaPollLimit;
  tc::Tables4 tc_tables{};   // the tensor-core form's matrices (precision BF16X3_TC)
  void* tc_owned = nullptr;
  bool tc_on = false;
  void use_tma() {
    TmaConfig& t = tma_config();
    t.err = tma_err;
    t.sms = sms;
    t.enabled = true;
    t.skip_tile = inject_skip;
    t.poll_limit = inject_polls;
    t.tc = tc_on ? &tc_tables : nullptr;
    t.tc_axes = 3;
    t.zwarp[0] = false;
    t.zwarp[1] = true;
  }
  void end_tma() {   // the injection lasts one execution
    TmaConfig& t = tma_config();
    t.tc = nullptr;
    t.skip_tile = inject_skip = -1;
    t.poll_limit = inject_polls = kTmaPollLimit;
  }
  // after a synchronised execution: did a tile wait give up?
  cudaError_t timed_out(bool* out) {
    int f = 0;
    cudaError_t e = cudaMemcpy(&f, tma_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && f) e = cudaMemset(tma_err, 0, sizeof(int));
    *out = f != 0;
    return e;
  }
};

template <typename T>
struct R2R : R2RBase {
  DevTwiddles<T> tw[3];
  AxisTables<T> tb{};
  int kind[3];
  ~R2R() override {
    cudaSetDevice(device);
    for (auto& t : tw) t.release();
    if (tc_owned) cudaFree(tc_owned);
    if (own) cudaStreamDestroy(own);
    if (tma_err) cudaFree(tma_err);
  }
  cudaError_t setup() {
    const int len[3] = {nx, ny, nz};
    cudaError_t e;
    for (int a = 0; a < 3; ++a) {
      if ((e = tw[a].upload(len[a])) != cudaSuccess) return e;
      tb.t[a] = tw[a].tables();
    }
    if ((e = cudaMalloc(&tma_err, sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMemset(tma_err, 0, sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
    return cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking);
  }
  cudaError_t exec(void* data, cudaStream_t s) override {
    T* d = static_cast<T*>(data);
    const Geom g{nx, ny, nz};
    cudaError_t e;
    use_tma();
    const int k3[3] = {kind[0], kind[1], kind[2]};
    e = yz3(g, tb, k3, d, StoreField<T>{g, d}, s);
    if (e == cudaSuccess) e = launch_pass<T, 0>(g, kind[0], tb.t[0], LoadField<T>{g, d}, StoreField<T>{g, d}, s);
    end_tma();
    return e;
  }
};

}  // namespace quasi

struct quasi_r2r_plan {
  quasi::R2RBase* impl;
};

// The r2r entry points report through the same quasi_last_error() as the rest
// of the ABI (abi.cu owns the per-thread message).
namespace quasi {
int set_error(int code, const std::string& msg);
}
using quasi::set_error;

extern "C" {

int quasi_r2r_plan_create(int nx, int ny, int nz, const int kind[3], int precision, int device,
                          quasi_r2r_plan** out) {
  if (!out || !kind) return set_error(QUASI_ERR_INVALID, "null argument");
  *out = nullptr;
  quasi_config c{};
  quasi_config_default(&c, QUASI_VARIANT_QUASI, nx, ny, nz);
  c.precision = precision;
  c.device = device;
  std::string why = quasi::validate_config(c);
  if (!why.empty()) return set_error(QUASI_ERR_INVALID, why.c_str());
  for (int a = 0; a < 3; ++a)
    if (kind[a] < 0 || kind[a] > 3)
      return set_error(QUASI_ERR_INVALID, "kind must be 0..3 (REDFT10 REDFT01 RODFT10 RODFT01)");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return set_error(QUASI_ERR_NODEVICE, "no CUDA device available (no CPU fallback)");
  }
  if (device < 0 || device >= count) return set_error(QUASI_ERR_INVALID, "device ordinal out of range");
  if (cudaSetDevice(device) != cudaSuccess) return set_error(QUASI_ERR_CUDA, "cudaSetDevice failed");
  quasi::R2RBase* b;
  cudaError_t e;
  if (precision == QUASI_PREC_FP64) {
    auto* p = new quasi::R2R<double>();
    p->nx = nx; p->ny = ny; p->nz = nz; p->device = device; p->elem = 8;
    for (int a = 0; a < 3; ++a) p->kind[a] = kind[a];
    e = p->setup();
    b = p;
  } else {
    auto* p = new quasi::R2R<float>();
    p->nx = nx; p->ny = ny; p->nz = nz; p->device = device; p->elem = 4;
    for (int a = 0; a < 3; ++a) p->kind[a] = kind[a];
    e = p->setup();
    if (e == cudaSuccess && precision == QUASI_PREC_BF16X3_TC) {
      e = quasi::tc::upload_tables(p->tc_tables, &p->tc_owned);
      p->tc_on = true;
    }
    b = p;
  }
  if (e != cudaSuccess) {
    delete b;
    return set_error(QUASI_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = new quasi_r2r_plan{b};
  return QUASI_OK;
}

int quasi_r2r_execute_device(quasi_r2r_plan* p, void* data, void* stream) {
  if (!p || !data) return set_error(QUASI_ERR_INVALID, "null argument");
  cudaSetDevice(p->impl->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->impl->own;
  cudaError_t e = p->impl->exec(data, s);
  if (e == cudaSuccess && !stream) e = cudaStreamSynchronize(s);
  bool late = false;
  if (e == cudaSuccess && !stream) e = p->impl->timed_out(&late);
  if (e != cudaSuccess) return set_error(QUASI_ERR_CUDA, cudaGetErrorString(e));
  if (late) return set_error(QUASI_ERR_TIMEOUT, "a tile copy did not complete within its wait limit");
  return QUASI_OK;
}

int quasi_r2r_execute_host(quasi_r2r_plan* p, const double* in, double* out) {
  if (!p || !in || !out) return set_error(QUASI_ERR_INVALID, "null argument");
  quasi::R2RBase* b = p->impl;
  cudaSetDevice(b->device);
  const size_t n = size_t(b->nx) * b->ny * b->nz;
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, n * b->elem);
  if (e != cudaSuccess) return set_error(QUASI_ERR_NOMEM, cudaGetErrorString(e));
  std::vector<float> f;
  if (b->elem == 8) {
    e = cudaMemcpyAsync(d, in, n * 8, cudaMemcpyHostToDevice, b->own);
  } else {
    f.assign(in, in + n);
    e = cudaMemcpyAsync(d, f.data(), n * 4, cudaMemcpyHostToDevice, b->own);
  }
  if (e == cudaSuccess) e = b->exec(d, b->own);
  if (e == cudaSuccess) {
    if (b->elem == 8) e = cudaMemcpyAsync(out, d, n * 8, cudaMemcpyDeviceToHost, b->own);
    else e = cudaMemcpyAsync(f.data(), d, n * 4, cudaMemcpyDeviceToHost, b->own);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->own);
  bool late = false;
  if (e == cudaSuccess) e = b->timed_out(&late);
  quasi::MapCache::get().forget(d, static_cast<char*>(d) + n * b->elem);
  cudaFree(d);
  if (e != cudaSuccess) return set_error(QUASI_ERR_CUDA, cudaGetErrorString(e));
  if (late) return set_error(QUASI_ERR_TIMEOUT, "a tile copy did not complete within its wait limit");
  if (b->elem == 4)
    for (size_t i = 0; i < n; ++i) out[i] = f[i];
  return QUASI_OK;
}

int quasi_r2r_inject_wait_timeout(quasi_r2r_plan* p, int skip_tile, unsigned poll_limit) {
  if (!p || skip_tile < 0 || poll_limit < 1) return set_error(QUASI_ERR_INVALID, "need a plan, skip_tile >= 0, poll_limit >= 1");
  p->impl->inject_skip = skip_tile;
  p->impl->inject_polls = poll_limit;
  return QUASI_OK;
}

int quasi_r2r_plan_destroy(quasi_r2r_plan* p) {
  if (!p) return QUASI_OK;
  delete p->impl;
  delete p;
  return QUASI_OK;
}

}  // extern "C"
