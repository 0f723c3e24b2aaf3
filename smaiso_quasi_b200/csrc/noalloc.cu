// quasi_diagnostics_noalloc: the FP64 diagnostics reduction (L1, mass,
// energy) for callers that cannot allocate device memory.
//
// Some callers of this library are not allowed to call cudaMalloc: code that
// runs while another component owns every byte of the device through its
// own pool (a solver embedded in a larger framework), a host loop with a
// real-time budget where an allocation's implicit synchronisation is not
// acceptable, or a process that is about to be checkpointed and must not
// grow its device footprint.  They hold the fields in their own device
// buffers and pass them in; this entry point needs no handle and allocates
// nothing.  Its scratch (the per-block partial sums) is a file-scope
// __device__ array of fixed size that every GPU loading the library keeps
// until the process exits.
//
// Limits and behaviour:
//   - grids of up to kNoAllocMaxBlocks * kCellsPerBlock = 2^25 cells
//     (e.g. 256^3 and 256x256x512); larger grids are rejected with an error;
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture;
//   - every call shares the one array: calls that overlap on the GPU (other
//     streams, other host threads) race.  Each call writes every slot it
//     reads, so nothing has to start at zero;
//   - the call runs on cfg->device (made current for the call, the caller's
//     current device restored afterwards) and rejects field pointers that are
//     not device memory of that device;
//   - the call waits for its stream and copies the sums to the host, so it
//     cannot be made on a stream that is being captured (it returns
//     QUASI_ERR_STATE there).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine_impl.cuh"

namespace quasi {
int set_error(int code, const std::string& msg);
}

namespace {

constexpr int kNoAllocMaxBlocks = 2048;
constexpr size_t kCellsPerBlock = size_t(quasi::kDiagThreads) * 64;   // 64 cells per thread
constexpr int kScratchDoubles = kNoAllocMaxBlocks * 4 + 4;              // partials, then the 4 sums

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_dev[256] = {};   // device address of g_noalloc_scratch, per device ordinal

// Set-up, once per device, with that device current.
int scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return quasi::set_error(QUASI_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 256) return quasi::set_error(QUASI_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return quasi::set_error(QUASI_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_dev[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_dev[dev];
  return QUASI_OK;
}

template <typename T>
cudaError_t reduce(const void* psi, const void* psi_old, const void* rho, const void* df, size_t n, int blocks,
                   double ep, const quasi_config& c, int energy, double* scratch, double* host4, cudaStream_t s) {
  quasi::diag_partial_kernel<T><<<blocks, quasi::kDiagThreads, 0, s>>>(
      static_cast<const T*>(psi), static_cast<const T*>(psi_old), static_cast<const T*>(rho),
      static_cast<const T*>(df), ep, c.alpha, c.beta, c.gamma, energy, n, scratch);
  quasi::diag_final_kernel<<<1, 32, 0, s>>>(scratch, blocks, scratch + kNoAllocMaxBlocks * 4);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(host4, scratch + kNoAllocMaxBlocks * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}

// Restores the caller's current device when the call returns.
struct DeviceScope {
  int prev = -1;
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// A field argument must be device memory of `device` (cudaPointerGetAttributes
// allocates nothing).
bool on_device(const void* p, int device) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice && a.device == device;
}

}  // namespace

extern "C" QUASI_API int quasi_diagnostics_noalloc(const quasi_config* cfg, const void* psi, const void* psi_old,
                                                   const void* rho, const void* df, double out[3], void* stream) {
  if (!cfg || !psi || !psi_old || !rho || !out) return quasi::set_error(QUASI_ERR_INVALID, "null argument");
  const int energy = cfg->variant == QUASI_VARIANT_QUASI;
  if (cfg->variant != QUASI_VARIANT_QUASI && cfg->variant != QUASI_VARIANT_STB)
    return quasi::set_error(QUASI_ERR_INVALID, "unknown variant");
  if (energy && !df) return quasi::set_error(QUASI_ERR_INVALID, "df is required for the quasi variant's energy");
  if (cfg->nx <= 0 || cfg->ny <= 0 || cfg->nz <= 0) return quasi::set_error(QUASI_ERR_INVALID, "bad grid");
  if (cfg->precision != QUASI_PREC_FP64 && cfg->precision != QUASI_PREC_FP32)
    return quasi::set_error(QUASI_ERR_INVALID, "unknown precision");
  // the same scalar checks as quasi_create: L1 divides by dt, dx needs q0 and nw
  if (!(cfg->dt > 0) || !(cfg->q0 > 0) || cfg->nw <= 0)
    return quasi::set_error(QUASI_ERR_INVALID, "dt, q0 and nw must be positive");
  const size_t n = size_t(cfg->nx) * cfg->ny * cfg->nz;
  const size_t blocks = (n + kCellsPerBlock - 1) / kCellsPerBlock;
  if (blocks > size_t(kNoAllocMaxBlocks))
    return quasi::set_error(QUASI_ERR_INVALID,
                            "grid of " + std::to_string(n) + " cells exceeds the static scratch of " +
                                std::to_string(kNoAllocMaxBlocks) + " partial sums (at most " +
                                std::to_string(size_t(kNoAllocMaxBlocks) * kCellsPerBlock) + " cells)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return quasi::set_error(QUASI_ERR_NODEVICE, "no CUDA device available (libquasi_gpu has no CPU fallback)");
  }
  if (cfg->device < 0 || cfg->device >= ndev) return quasi::set_error(QUASI_ERR_INVALID, "device ordinal out of range");
  DeviceScope scope;
  cudaError_t e = cudaGetDevice(&scope.prev);
  if (e != cudaSuccess) return quasi::set_error(QUASI_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (scope.prev == cfg->device) scope.prev = -1;   // nothing to restore
  else if ((e = cudaSetDevice(cfg->device)) != cudaSuccess)
    return quasi::set_error(QUASI_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  const void* fields[4] = {psi, psi_old, rho, energy ? df : psi};
  for (const void* f : fields)
    if (!on_device(f, cfg->device))
      return quasi::set_error(QUASI_ERR_INVALID, "a field pointer is not device memory of cfg->device");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing(s, &cap)) != cudaSuccess)
    return quasi::set_error(QUASI_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  if (cap != cudaStreamCaptureStatusNone)
    return quasi::set_error(QUASI_ERR_STATE, "the call synchronises its stream: not allowed while it is captured");
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  const double ep = -0.001 * cfg->ep_arg;   // quasi.cpp:187
  double r[4];
  e = cfg->precision == QUASI_PREC_FP64
                      ? reduce<double>(psi, psi_old, rho, df ? df : rho, n, int(blocks), ep, *cfg, energy, scratch, r, s)
                      : reduce<float>(psi, psi_old, rho, df ? df : rho, n, int(blocks), ep, *cfg, energy, scratch, r, s);
  if (e != cudaSuccess) return quasi::set_error(QUASI_ERR_CUDA, cudaGetErrorString(e));
  const double dx = (cfg->nx * 2.0 * M_PI / (cfg->q0 * cfg->nw)) / cfg->nx;
  out[0] = r[0] / (cfg->dt * r[1]);
  out[1] = r[2] * dx * dx * dx;
  out[2] = energy ? r[3] * dx * dx * dx : 0.0;
  return QUASI_OK;
}
