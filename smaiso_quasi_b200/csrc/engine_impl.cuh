// Engine<T>: one simulation instance on one GPU.  Included by engine_f64.cu
// and engine_f32.cu, which instantiate it for double and float.
#pragma once
#include <cstdint>
#include <fstream>
#include <mutex>

#include "engine.cuh"

namespace quasi {

// ---------------------------------------------------------------------------
// FP64 reductions: L1 numerator/denominator, mass, energy (quasi.cpp:1983-1996)
// ---------------------------------------------------------------------------
constexpr int kDiagBlocks = 592;   // 4 x 148 SMs
constexpr int kDiagThreads = 256;

// P: the type of psi and psi_old, R: of rho, F: of df (the engine holds psi
// and rho in double; the allocation-free entry point takes one type for all)
template <typename P, typename R = P, typename F = P>
__global__ void __launch_bounds__(kDiagThreads) diag_partial_kernel(const P* psi, const P* psi_old, const R* rho,
                                                                    const F* df, double ep, double alpha, double beta,
                                                                    double gamma, int with_energy, size_t n,
                                                                    double* partial) {
  double a = 0, b = 0, m = 0, en = 0;
  for (size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x; id < n; id += size_t(gridDim.x) * blockDim.x) {
    const double ps = psi[id];
    a += fabs(ps - double(psi_old[id]));
    b += fabs(ps);
    const double r = rho[id];
    m += r;
    if (with_energy) {
      const double d = df[id], p2 = ps * ps;
      en += r * (-0.5 * ep * p2 + 0.5 * alpha * d * d - 0.25 * beta * p2 * p2 + (gamma / 6) * p2 * p2 * p2);
    }
  }
  __shared__ double red[4][kDiagThreads / 32];
  double v[4] = {a, b, m, en};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int w = 0; w < kDiagThreads / 32; ++w) s += red[threadIdx.x][w];
    partial[blockIdx.x * 4 + threadIdx.x] = s;
  }
}

static __global__ void diag_final_kernel(const double* partial, int nblocks, double* out) {
  // fixed-order sums: deterministic run to run
  if (threadIdx.x < 4) {
    double s = 0;
    for (int b = 0; b < nblocks; ++b) s += partial[b * 4 + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

template <typename T>
class Engine : public EngineBase {
 public:
  // fields of the storage type (+ the float copies of psiq and rhoq); then
  // the double fields: psiq x 3, rhoq, rho, rho_old, psi x 2, grad psi x 3
  // (+ the scratch of the double transforms in the FP32 form)
  // FP32: + the float copies of psi^, rho^; FP64: + the second grad rho buffers
  static constexpr int kFields = 22 + (kStateCopy<T> ? 2 : 3);
  static constexpr int kDFields = 11 + (kStateCopy<T> ? 1 : 0);
  static constexpr int kPhases = 6;   // lcm of the 3-buffer psiq and 2-buffer Nq rotations

  explicit Engine(const quasi_config& cfg) : cfg_(cfg) {}

  ~Engine() override {
    if (dev_ok_) cudaSetDevice(cfg_.device);
    for (auto& ge : graph_exec_)
      if (ge) cudaGraphExecDestroy(ge);
    for (auto& gr : graph_)
      if (gr) cudaGraphDestroy(gr);
    if (slab_) {
      MapCache::get().forget(slab_, static_cast<char*>(slab_) + size_t(kFields) * n_ * sizeof(T));
      cudaFree(slab_);
    }
    if (dslab_) {
      MapCache::get().forget(dslab_, dslab_ + size_t(kDFields) * n_);
      cudaFree(dslab_);
    }
    for (auto& t : tw64_) t.release();
    if (tc_owned_) cudaFree(tc_owned_);
    if (tma_err_) cudaFree(tma_err_);
    if (tabs_) cudaFree(tabs_);
    if (nloop_dev_) cudaFree(nloop_dev_);
    if (partial_) cudaFree(partial_);
    if (host_stage_) cudaFreeHost(host_stage_);
    for (auto& t : tw_) t.release();
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    for (auto& e : fork_ev_)
      if (e) cudaEventDestroy(e);
    if (stream2_) cudaStreamDestroy(stream2_);
    if (stream_) cudaStreamDestroy(stream_);
  }

  int create() {
    if (!cuda_ok(cudaSetDevice(cfg_.device), "cudaSetDevice")) return QUASI_ERR_NODEVICE;
    dev_ok_ = true;
    g_ = Geom{cfg_.nx, cfg_.ny, cfg_.nz};
    n_ = size_t(g_.nx) * g_.ny * g_.nz;
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream")) return QUASI_ERR_CUDA;
    // second capture stream and fork/join events of the step graphs
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking), "stream")) return QUASI_ERR_CUDA;
    for (auto& e : fork_ev_)
      if (!cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event")) return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaEventCreate(&ev0_), "event") || !cuda_ok(cudaEventCreate(&ev1_), "event")) return QUASI_ERR_CUDA;
    const size_t bytes = size_t(kFields) * n_ * sizeof(T), dbytes = size_t(kDFields) * n_ * sizeof(double);
    if (cudaMalloc(&slab_, bytes) != cudaSuccess || cudaMalloc(&dslab_, dbytes) != cudaSuccess) {
      cudaGetLastError();
      err = "device allocation of " + std::to_string(bytes + dbytes) + " bytes failed";
      return QUASI_ERR_NOMEM;
    }
    if (!cuda_ok(cudaMemset(slab_, 0, bytes), "memset") || !cuda_ok(cudaMemset(dslab_, 0, dbytes), "memset"))
      return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaMalloc(&nloop_dev_, sizeof(int)), "malloc") || !cuda_ok(cudaMemset(nloop_dev_, 0, sizeof(int)), "memset"))
      return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaMalloc(&partial_, (kDiagBlocks * 4 + 4) * sizeof(double)), "malloc")) return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaMalloc(&tma_err_, sizeof(int)), "malloc") || !cuda_ok(cudaMemset(tma_err_, 0, sizeof(int)), "memset"))
      return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, cfg_.device), "attribute"))
      return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaMallocHost(&host_stage_, n_ * sizeof(double) + 64), "host alloc")) return QUASI_ERR_NOMEM;
    // wavenumber tables, quasi.cpp:397-431
    const int len[3] = {g_.nx, g_.ny, g_.nz};
    std::vector<double> h;
    for (int a = 0; a < 3; ++a) {
      const int n = len[a];
      const double L = n * 2.0 * M_PI / (cfg_.q0 * cfg_.nw);
      const double d = L / n;
      for (int i = 0; i < n; ++i) h.push_back(1.0 * M_PI * i / (d * n));
      for (int i = 0; i < n; ++i) h.push_back(1.0 * M_PI * (i + 1) / (d * n));
    }
    // then the density filter per axis, exp(-1.57^2 8 vq^2) (quasi.cpp:1260)
    for (int a = 0, off = 0; a < 3; off += 2 * len[a], ++a)
      for (int i = 0; i < len[a]; ++i) h.push_back(std::exp(-1.57 * 1.57 * 8 * h[off + i] * h[off + i]));
    if (!cuda_ok(cudaMalloc(&tabs_, h.size() * sizeof(double)), "malloc")) return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaMemcpy(tabs_, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice), "memcpy"))
      return QUASI_ERR_CUDA;
    for (int a = 0; a < 3; ++a)
      if (!cuda_ok(tw_[a].upload(len[a]), "twiddles")) return QUASI_ERR_CUDA;
    for (int a = 0; a < 3; ++a) tb_.t[a] = tw_[a].tables();
    if (cfg_.precision == QUASI_PREC_BF16X3_TC) {   // the tensor-core form's matrices
      if (!cuda_ok(tc::upload_tables(tc_tables_, &tc_owned_), "contraction matrices")) return QUASI_ERR_CUDA;
      tc_on_ = true;
    }
    if constexpr (kStateCopy<T>) {   // the double transforms' own tables
      for (int a = 0; a < 3; ++a)
        if (!cuda_ok(tw64_[a].upload(len[a]), "twiddles")) return QUASI_ERR_CUDA;
      for (int a = 0; a < 3; ++a) tb64_.t[a] = tw64_[a].tables();
    } else {
      for (int a = 0; a < 3; ++a)
        tb64_.t[a] = Tables<double>{reinterpret_cast<const Cx<double>*>(tb_.t[a].root),
                                    reinterpret_cast<const Cx<double>*>(tb_.t[a].quarter)};
    }
    build_ctx(h);
    if (!layout_ok_) { err = "internal error: field layout does not match the slab sizes"; return QUASI_ERR_CUDA; }
    // the six step graphs are made here, like the reference's FFTW plans
    // before its loop: quasi_step only launches them
    if (cfg_.autotune == 1) {
      const int rc = autotune();
      if (rc) return rc;
    } else if (cfg_.autotune == 2) {   // every warp-tile candidate (tests of those kernels)
      tune_.zwarp[0] = tune_.zwarp[1] = true;
      for (auto& a : tune_.xywarp) a[0] = a[1] = true;
    }
    return capture();
  }

  // Time each tunable pass's candidate kernels on the scratch fields (zeros)
  // and keep the fastest: the z pass as CTA or warp tiles, per type; in the
  // BF16X3 form the plain x and y passes on the tensor cores or by FFT.  The
  // two candidates are timed in alternation (5 rounds of 10 launches each, the
  // best round of each counts), and the default stays unless the other is
  // faster by more than 3%.  The choices are kept per (device, grid, form) for
  // the handles created later in the process (an ensemble's members of one
  // grid tune once).
  int autotune() {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int>, Tuning> cache;
    const auto key = std::make_tuple(cfg_.device, g_.nx, g_.ny, g_.nz, cfg_.precision);
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = cache.find(key);
      if (it != cache.end()) {
        tune_ = it->second;
        return QUASI_OK;
      }
    }
    // *ms < 0: the candidate does not cover this shape (the step uses the
    // general kernel there), nothing to choose
    auto time = [&](auto&& launch, float* ms) -> bool {
      const cudaError_t e0 = launch();
      if (e0 == cudaErrorNotSupported) {
        *ms = -1;
        return true;
      }
      if (!cuda_ok(e0, "autotune")) return false;
      if (!cuda_ok(cudaEventRecord(ev0_, stream_), "event")) return false;
      for (int r = 0; r < 10; ++r)
        if (!cuda_ok(launch(), "autotune")) return false;
      if (!cuda_ok(cudaEventRecord(ev1_, stream_), "event") || !cuda_ok(cudaEventSynchronize(ev1_), "sync"))
        return false;
      return cuda_ok(cudaEventElapsedTime(ms, ev0_, ev1_), "elapsed");
    };
    // best[v] over alternating rounds of the two settings applied by set(v)
    auto race = [&](auto&& set, auto&& launch, float best[2]) -> bool {
      best[0] = best[1] = 1e30f;
      for (int round = 0; round < 5; ++round)
        for (int v = 0; v < 2; ++v) {
          set(v);
          use_tma();
          float ms = 0;
          if (!time(launch, &ms)) return false;
          if (ms < 0) {
            best[0] = best[1] = -1;
            return true;
          }
          best[v] = std::min(best[v], ms);
        }
      return true;
    };
    auto better = [](const float ms[2], bool dflt) {   // the chosen setting
      if (ms[0] < 0 || ms[1] < 0) return dflt;
      const float cur = ms[dflt ? 1 : 0], alt = ms[dflt ? 0 : 1];
      return alt < 0.97f * cur ? !dflt : dflt;
    };
    Tuning best = tune_;
    // z pass, storage type and (FP32 form) double
    for (int d = 0; d < (kStateCopy<T> ? 2 : 1); ++d) {
      const int slot = kStateCopy<T> ? d : 1;
      float ms[2];
      auto z = [&]() -> cudaError_t {
        if (d == 0) return launch_zpass<T>(g_, E01, tb_.t[2], c_.tmp, c_.tmp, stream_);
        return launch_zpass<double>(g_, E01, tb64_.t[2], c_.tmp64, c_.tmp64, stream_);
      };
      if (!race([&](int v) { tune_.zwarp[slot] = v == 1; }, z, ms)) return QUASI_ERR_CUDA;
      best.zwarp[slot] = better(ms, Tuning{}.zwarp[slot]);
      tune_ = best;
      // x and y passes as CTA or warp tiles (the plain pass decides for all
      // passes of that axis and type)
      for (int a = 0; a < 2; ++a) {
        auto xy = [&]() -> cudaError_t {
          if (d == 0) {
            if (a == 0) return launch_pass<T, 0>(g_, E01, tb_.t[0], LoadField<T>{g_, c_.tmp}, StoreField<T>{g_, c_.tmp}, stream_);
            return launch_pass<T, 1>(g_, E01, tb_.t[1], LoadField<T>{g_, c_.tmp}, StoreField<T>{g_, c_.tmp}, stream_);
          }
          if (a == 0)
            return launch_pass<double, 0>(g_, E01, tb64_.t[0], LoadField<double>{g_, c_.tmp64},
                                          StoreField<double>{g_, c_.tmp64}, stream_);
          return launch_pass<double, 1>(g_, E01, tb64_.t[1], LoadField<double>{g_, c_.tmp64},
                                        StoreField<double>{g_, c_.tmp64}, stream_);
        };
        const int tc_keep = tune_.tc_axes;
        tune_.tc_axes = 0;   // the FFT passes are what is tuned here
        if (!race([&](int v) { tune_.xywarp[a][slot] = v == 1; }, xy, ms)) return QUASI_ERR_CUDA;
        tune_.tc_axes = tc_keep;
        best.xywarp[a][slot] = better(ms, false);
        tune_ = best;
      }
    }
    if (tc_on_) {   // x (bit 0) and y (bit 1) on the tensor cores or by FFT
      int axes = 0;
      for (int a = 0; a < 2; ++a) {
        float ms[2];
        auto p = [&]() -> cudaError_t {
          if (a == 0) return launch_pass<T, 0>(g_, E01, tb_.t[0], LoadField<T>{g_, c_.tmp}, StoreField<T>{g_, c_.tmp}, stream_);
          return launch_pass<T, 1>(g_, E01, tb_.t[1], LoadField<T>{g_, c_.tmp}, StoreField<T>{g_, c_.tmp}, stream_);
        };
        if (!race([&](int v) { tune_.tc_axes = v ? (1 << a) : 0; }, p, ms)) return QUASI_ERR_CUDA;
        if (better(ms, true)) axes |= 1 << a;
      }
      best.tc_axes = axes;
    }
    best.measured = true;
    tune_ = best;
    std::lock_guard<std::mutex> lk(mu);
    cache.emplace(key, best);
    return QUASI_OK;
  }

  int set_psi(const double* host) override {
    set_phase(0);   // quasi_init starts the rotation at phase 0
    double* st = static_cast<double*>(host_stage_);
    bool finite = true;
    std::mutex mu;
    host_parallel(n_, [&](size_t lo, size_t hi) {
      bool ok = true;
      for (size_t i = lo; i < hi; ++i) {
        st[i] = host[i];
        ok = ok && std::isfinite(host[i]);
      }
      if (!ok) {
        std::lock_guard<std::mutex> lk(mu);
        finite = false;
      }
    });
    if (!finite) { err = "initial psi has a NaN or infinite value"; return QUASI_ERR_INVALID; }
    if (!cuda_ok(cudaMemcpyAsync(c_.psi, st, n_ * sizeof(double), cudaMemcpyHostToDevice, stream_), "H2D"))
      return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(stream_), "sync")) return QUASI_ERR_CUDA;
    have_psi_ = true;
    initialized_ = false;
    return QUASI_OK;
  }

  int init() override {
    if (!have_psi_) { err = "quasi_init before quasi_set_psi"; return QUASI_ERR_STATE; }
    set_phase(0);
    use_tma();
    if (!cuda_ok(enqueue_init<T>(c_, tb_, tb64_, nloop_dev_, stream_), "init")) return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(stream_), "init sync")) return QUASI_ERR_CUDA;
    nloop_ = 0;
    initialized_ = true;
    return QUASI_OK;
  }

  int step(int nsteps, double* device_ms) override {
    int rc = enqueue(nsteps, device_ms != nullptr);
    if (rc) return rc;
    rc = synchronize();
    if (rc) return rc;
    if (device_ms) {
      float ms = 0;
      if (!cuda_ok(cudaEventElapsedTime(&ms, ev0_, ev1_), "elapsed")) return QUASI_ERR_CUDA;
      *device_ms = ms;
    }
    return QUASI_OK;
  }

  int step_async(int nsteps) override { return enqueue(nsteps, false); }

  int synchronize() override {
    if (!cuda_ok(cudaStreamSynchronize(stream_), "step sync")) return QUASI_ERR_CUDA;
    int tma_failed = 0;
    if (!cuda_ok(cudaMemcpy(&tma_failed, tma_err_, sizeof(int), cudaMemcpyDeviceToHost), "flag")) return QUASI_ERR_CUDA;
    if (tma_failed) {
      cudaMemset(tma_err_, 0, sizeof(int));
      err = "a tile copy did not complete within its wait limit";
      return QUASI_ERR_TIMEOUT;
    }
    return QUASI_OK;
  }

  int get_field(int field, double* host) override {
    set_phase(nloop_);
    const Field f = field_ptr(field);
    if (!f.p) { err = "unknown or unavailable field " + std::to_string(field); return QUASI_ERR_INVALID; }
    if (!cuda_ok(cudaMemcpyAsync(host_stage_, f.p, n_ * f.elem, cudaMemcpyDeviceToHost, stream_), "D2H"))
      return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(stream_), "sync")) return QUASI_ERR_CUDA;
    host_parallel(n_, [&](size_t lo, size_t hi) {
      if (f.elem == sizeof(double)) {
        std::memcpy(host + lo, static_cast<const double*>(host_stage_) + lo, (hi - lo) * sizeof(double));
      } else {
        const float* st = static_cast<const float*>(host_stage_);
        for (size_t i = lo; i < hi; ++i) host[i] = double(st[i]);
      }
    });
    return QUASI_OK;
  }

  int diagnostics(double out[3]) override {
    if (!initialized_) { err = "diagnostics before quasi_init"; return QUASI_ERR_STATE; }
    const int energy = cfg_.variant == QUASI_VARIANT_QUASI;
    set_phase(nloop_);
    diag_partial_kernel<double, double, T><<<kDiagBlocks, kDiagThreads, 0, stream_>>>(
        c_.psi, c_.psi_old, c_.rho, c_.df, c_.ep, c_.alpha, c_.beta, c_.gamma, energy, n_, partial_);
    diag_final_kernel<<<1, 32, 0, stream_>>>(partial_, kDiagBlocks, partial_ + kDiagBlocks * 4);
    double r[4];
    if (!cuda_ok(cudaMemcpyAsync(r, partial_ + kDiagBlocks * 4, sizeof(r), cudaMemcpyDeviceToHost, stream_), "D2H"))
      return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(stream_), "sync")) return QUASI_ERR_CUDA;
    const double dx = (g_.nx * 2.0 * M_PI / (cfg_.q0 * cfg_.nw)) / g_.nx;
    out[0] = r[0] / (c_.dt * r[1]);
    out[1] = r[2] * dx * dx * dx;
    out[2] = energy ? r[3] * dx * dx * dx : 0.0;
    return QUASI_OK;
  }

  int growth_rate(double* out) override {
    const double vq1 = M_PI * 1 / ((g_.nz * 2.0 * M_PI / (cfg_.q0 * cfg_.nw)) / g_.nz * g_.nz);
    const int i = (int)std::lround(cfg_.q_pert / vq1), k = (int)std::lround(cfg_.q0 / vq1);
    if (i < 0 || i >= g_.nx || k < 0 || k >= g_.nz) { err = "growth probe mode outside the grid"; return QUASI_ERR_INVALID; }
    const size_t id = (size_t(i) * g_.ny + 0) * g_.nz + k;
    double a, b;
    set_phase(nloop_);
    if (!cuda_ok(cudaMemcpyAsync(&a, c_.psiq + id, sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H") ||
        !cuda_ok(cudaMemcpyAsync(&b, c_.psiq_old + id, sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H") ||
        !cuda_ok(cudaStreamSynchronize(stream_), "sync"))
      return QUASI_ERR_CUDA;
    *out = (a - b) / (cfg_.dt * b);
    return QUASI_OK;
  }

  // Binary checkpoint: header + the carried state (each field in its own
  // type) + a checksum of everything after the header.
  int save(const char* path) override {
    if (!initialized_) { err = "save before quasi_init"; return QUASI_ERR_STATE; }
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = std::string("cannot open ") + path; return QUASI_ERR_IO; }
    Header hd = header();
    f.write(reinterpret_cast<const char*>(&hd), sizeof(hd));
    set_phase(nloop_);
    uint64_t sum = kCheckSeed;
    for (const Field& fd : carried()) {
      if (!cuda_ok(cudaMemcpy(host_stage_, fd.p, n_ * fd.elem, cudaMemcpyDeviceToHost), "D2H")) return QUASI_ERR_CUDA;
      sum = checksum(sum, host_stage_, n_ * fd.elem);
      f.write(static_cast<const char*>(host_stage_), n_ * fd.elem);
    }
    f.write(reinterpret_cast<const char*>(&sum), sizeof(sum));
    if (!f) { err = std::string("write failed: ") + path; return QUASI_ERR_IO; }
    return QUASI_OK;
  }

  int load(const char* path) override {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = std::string("cannot open ") + path; return QUASI_ERR_IO; }
    Header hd{}, want = header();
    f.read(reinterpret_cast<char*>(&hd), sizeof(hd));
    if (!f || std::memcmp(hd.magic, want.magic, 8) != 0) { err = "not a quasi checkpoint"; return QUASI_ERR_IO; }
    if (hd.nx != want.nx || hd.ny != want.ny || hd.nz != want.nz || hd.variant != want.variant ||
        hd.elem != want.elem) {
      err = "checkpoint grid/variant/precision does not match the handle";
      return QUASI_ERR_IO;
    }
    if (hd.nloop < 0) { err = "checkpoint step count is negative"; return QUASI_ERR_IO; }
    // verify the whole file (length and checksum) before any of it reaches
    // the device, so that a failed load leaves the handle as it was; then
    // read it again field by field
    const std::vector<Field> fields = carried_at(hd.nloop);
    uint64_t sum = kCheckSeed;
    for (const Field& fd : fields) {
      f.read(static_cast<char*>(host_stage_), std::streamsize(n_ * fd.elem));
      if (!f) { err = "checkpoint is truncated"; return QUASI_ERR_IO; }
      sum = checksum(sum, host_stage_, n_ * fd.elem);
    }
    uint64_t stored = 0;
    f.read(reinterpret_cast<char*>(&stored), sizeof(stored));
    if (!f) { err = "checkpoint is truncated"; return QUASI_ERR_IO; }
    if (f.peek() != std::char_traits<char>::eof()) { err = "checkpoint has trailing bytes"; return QUASI_ERR_IO; }
    if (sum != stored) { err = "checkpoint checksum mismatch (corrupt file)"; return QUASI_ERR_IO; }
    f.clear();
    f.seekg(sizeof(Header));
    for (const Field& fd : fields) {
      f.read(static_cast<char*>(host_stage_), std::streamsize(n_ * fd.elem));
      if (!f) { err = "checkpoint read failed"; return QUASI_ERR_IO; }
      if (!cuda_ok(cudaMemcpy(const_cast<void*>(fd.p), host_stage_, n_ * fd.elem, cudaMemcpyHostToDevice), "H2D"))
        return QUASI_ERR_CUDA;
    }
    set_phase(hd.nloop);
    int nl = int(hd.nloop);
    if (!cuda_ok(cudaMemcpy(nloop_dev_, &nl, sizeof(int), cudaMemcpyHostToDevice), "H2D")) return QUASI_ERR_CUDA;
    nloop_ = hd.nloop;
    have_psi_ = initialized_ = true;
    return QUASI_OK;
  }

  long nloop() const override { return nloop_; }
  cudaGraph_t phase_graph(int ph) const override { return graph_[ph]; }
  int phases() const override { return kPhases; }
  int device() const override { return cfg_.device; }
  void note_steps(int n) override { nloop_ += n; }
  bool initialized() const override { return initialized_; }
  void tuning(int out[4]) const override {
    for (int d = 0; d < 2; ++d)
      out[d] = int(tune_.zwarp[d]) | (int(tune_.xywarp[0][d]) << 1) | (int(tune_.xywarp[1][d]) << 2);
    out[2] = tc_on_ ? tune_.tc_axes : 0;
    out[3] = tune_.measured;
  }

  int step_kernels(int* n) override {
    if (!graph_exec_[0]) {
      if (!initialized_) { err = "step graph not captured yet (call quasi_init)"; return QUASI_ERR_STATE; }
      int rc = capture();
      if (rc) return rc;
    }
    *n = graph_kernels_;
    return QUASI_OK;
  }

  int time_axis_pass(int axis, int reps, double* avg_ms) override {
    if (axis < 0 || axis > 2 || reps < 1) { err = "axis must be 0..2 and reps >= 1"; return QUASI_ERR_INVALID; }
    T* d = c_.tmp;
    use_tma();
    auto one = [&]() -> cudaError_t {
      if (axis == 0) return launch_pass<T, 0>(g_, E01, tb_.t[0], LoadField<T>{g_, d}, StoreField<T>{g_, d}, stream_);
      if (axis == 1) return launch_pass<T, 1>(g_, E01, tb_.t[1], LoadField<T>{g_, d}, StoreField<T>{g_, d}, stream_);
      const cudaError_t e = launch_zpass<T>(g_, E01, tb_.t[2], d, d, stream_);
      if (e != cudaErrorNotSupported) return e;
      return launch_pass<T, 2>(g_, E01, tb_.t[2], LoadField<T>{g_, d}, StoreField<T>{g_, d}, stream_);
    };
    if (!cuda_ok(one(), "pass")) return QUASI_ERR_CUDA;   // warm
    if (!cuda_ok(cudaEventRecord(ev0_, stream_), "event")) return QUASI_ERR_CUDA;
    for (int r = 0; r < reps; ++r)
      if (!cuda_ok(one(), "pass")) return QUASI_ERR_CUDA;
    if (!cuda_ok(cudaEventRecord(ev1_, stream_), "event") || !cuda_ok(cudaEventSynchronize(ev1_), "sync"))
      return QUASI_ERR_CUDA;
    float ms = 0;
    if (!cuda_ok(cudaEventElapsedTime(&ms, ev0_, ev1_), "elapsed")) return QUASI_ERR_CUDA;
    *avg_ms = double(ms) / reps;
    return QUASI_OK;
  }

 private:
  struct Header {
    char magic[8];
    int32_t nx, ny, nz, variant, elem, pad;
    int64_t nloop;
  };
  // FNV-1a over 64-bit words (field sizes are multiples of 64 bytes)
  static constexpr uint64_t kCheckSeed = 1469598103934665603ull;
  static uint64_t checksum(uint64_t h, const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i + 8 <= n; i += 8) {
      uint64_t w;
      std::memcpy(&w, b + i, 8);
      h = (h ^ w) * 1099511628211ull;
    }
    return h;
  }
  Header header() const {
    Header h{};
    std::memcpy(h.magic, "QUASICK3", 8);
    h.nx = g_.nx; h.ny = g_.ny; h.nz = g_.nz; h.variant = cfg_.variant; h.elem = int(sizeof(T));
    h.nloop = nloop_;
    return h;
  }
  // Launch the step graphs of nsteps steps on the handle's stream (the host
  // step counter advances at once; the device one as the graphs run).
  int enqueue(int nsteps, bool timed) {
    if (!initialized_) { err = "quasi_step before quasi_init"; return QUASI_ERR_STATE; }
    if (nsteps < 0) { err = "nsteps < 0"; return QUASI_ERR_INVALID; }
    if (!graph_exec_[0]) {
      int rc = capture();
      if (rc) return rc;
    }
    if (timed && !cuda_ok(cudaEventRecord(ev0_, stream_), "event")) return QUASI_ERR_CUDA;
    for (int s = 0; s < nsteps; ++s)
      if (!cuda_ok(cudaGraphLaunch(graph_exec_[(nloop_ + s) % kPhases], stream_), "graph launch"))
        return QUASI_ERR_CUDA;
    if (timed && !cuda_ok(cudaEventRecord(ev1_, stream_), "event")) return QUASI_ERR_CUDA;
    nloop_ += nsteps;
    return QUASI_OK;
  }

  struct Field {
    const void* p;
    size_t elem;
  };
  // the state a step reads (at the phase set by set_phase(nloop))
  std::vector<Field> carried() {
    const size_t t = sizeof(T), d = sizeof(double);
    std::vector<Field> v = {{c_.psiq, d}, {c_.psiq_old, d}, {c_.Nq_old, t}, {c_.rhoq, d},  {c_.rho_old, d},
                            {c_.rho, d},  {c_.vx, t},       {c_.vy, t},     {c_.vz, t},    {c_.divv, t},
                            {c_.divvq, t}, {c_.psi, d},     {c_.psi_old, d}, {c_.p, t},    {c_.df, t},
                            {c_.gx, d},    {c_.gy, d},      {c_.gz, d}};
    if constexpr (kStateCopy<T>) {
      v.push_back({c_.psiq_t, t});
      v.push_back({c_.rhoq_t, t});
    } else {   // grad rho, computed by the previous step
      v.push_back({c_.rdx, t});
      v.push_back({c_.rdy, t});
      v.push_back({c_.rdz, t});
    }
    return v;
  }
  std::vector<Field> carried_at(long s) {
    const long keep = nloop_;
    set_phase(s);
    std::vector<Field> v = carried();
    set_phase(keep);
    return v;
  }

  // Buffer rotation for a step that starts after `s` completed steps:
  // psiq = A[s%3], psiq_old = A[(s+2)%3], psiq_new = A[(s+1)%3];
  // Nq (computed this step) = B[s%2], Nq_old = B[(s+1)%2];
  // psi = C[s%2], psi_old = psi_new = C[(s+1)%2] (psi_old is read only by the
  // diagnostics after the step, when it is C[s%2] again);
  // FP64 form: grad rho read = R[s%2], grad rho for the next step = R[(s+1)%2].
  void set_phase(long s) {
    c_.psiq = psiq_buf_[s % 3];
    c_.psiq_old = psiq_buf_[(s + 2) % 3];
    c_.psiq_new = psiq_buf_[(s + 1) % 3];
    if constexpr (!kStateCopy<T>) {   // the FP64 form reads the state itself
      c_.psiq_t = reinterpret_cast<T*>(c_.psiq);
      c_.rhoq_t = reinterpret_cast<T*>(c_.rhoq);
    }
    c_.Nq = nq_buf_[s % 2];
    c_.Nq_old = nq_buf_[(s + 1) % 2];
    c_.psi = psi_buf_[s % 2];
    c_.psi_old = psi_buf_[(s + 1) % 2];
    c_.psi_new = psi_buf_[(s + 1) % 2];
    // grad rho (the FP32 form has one buffer and no next)
    T* const* rd = rd_buf_[kStateCopy<T> ? 0 : s % 2];
    c_.rdx = rd[0]; c_.rdy = rd[1]; c_.rdz = rd[2];
    if constexpr (!kStateCopy<T>) {
      T* const* rn = rd_buf_[(s + 1) % 2];
      c_.rdnx = rn[0]; c_.rdny = rn[1]; c_.rdnz = rn[2];
    } else {
      c_.rdnx = c_.rdny = c_.rdnz = nullptr;
    }
  }

  void use_tma() {
    TmaConfig& t = tma_config();
    t.err = tma_err_;
    t.sms = sms_;
    t.enabled = true;
    t.tc = tc_on_ ? &tc_tables_ : nullptr;
    t.tc_axes = tune_.tc_axes;
    t.zwarp[0] = tune_.zwarp[0];
    t.zwarp[1] = tune_.zwarp[1];
    for (int a = 0; a < 2; ++a)
      for (int d = 0; d < 2; ++d) t.xywarp[a][d] = tune_.xywarp[a][d];
  }

  bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  }

  void build_ctx(const std::vector<double>& h) {
    T* f = static_cast<T*>(slab_);
    auto next = [&]() { T* p = f; f += n_; return p; };
    c_.g = g_;
    const double* t = tabs_;
    c_.vqx = t;                 c_.vsx = t + g_.nx;
    c_.vqy = t + 2 * g_.nx;     c_.vsy = c_.vqy + g_.ny;
    c_.vqz = t + 2 * g_.nx + 2 * g_.ny; c_.vsz = c_.vqz + g_.nz;
    const double* ft = t + 2 * (g_.nx + g_.ny + g_.nz);
    c_.fx = ft;
    c_.fy = ft + g_.nx;
    c_.fz = ft + g_.nx + g_.ny;
    (void)h;
    const bool quasi = cfg_.variant == QUASI_VARIANT_QUASI;
    c_.ep = -0.001 * cfg_.ep_arg;                                   // quasi.cpp:187
    c_.alpha = cfg_.alpha; c_.beta = cfg_.beta; c_.gamma = cfg_.gamma; c_.q0 = cfg_.q0;
    c_.kp = cfg_.kp; c_.rho0 = cfg_.rho_0;
    c_.rho_s = cfg_.kp * cfg_.amp + cfg_.rho_0;                     // quasi.cpp:197
    c_.rho_m = cfg_.rho_m > 0 ? cfg_.rho_m : c_.rho_s / 2;          // quasi.cpp:198
    c_.nu = quasi ? cfg_.nu_arg : 0.1 * cfg_.nu_arg;                // quasi.cpp:192, quasi-stb.cpp:191
    c_.dt = cfg_.dt;
    c_.scale = 0.125 / (double(g_.nx) * g_.ny * g_.nz);              // quasi.cpp:219
    c_.variant = cfg_.variant;
    c_.divv_switch = cfg_.divv_switch;
    c_.n0 = g_.nx / (cfg_.emulate_ranks > 0 ? cfg_.emulate_ranks : 1);
    c_.nloop = nloop_dev_;
    c_.store_dtpsi = quasi ? 0 : 1;
    double* dfp = dslab_;
    auto dnext = [&]() { double* p = dfp; dfp += n_; return p; };
    for (auto& b : psiq_buf_) b = dnext();
    c_.rhoq = dnext();
    c_.rho = dnext(); c_.rho_old = dnext();
    for (auto& b : psi_buf_) b = dnext();
    c_.gx = dnext(); c_.gy = dnext(); c_.gz = dnext();
    for (auto& b : nq_buf_) b = next();
    if constexpr (kStateCopy<T>) {
      c_.psiq_t = next();
      c_.rhoq_t = next();
    }
    c_.divvq = next(); c_.Sx = next(); c_.Sy = next(); c_.Sz = next();
    c_.vx = next(); c_.vy = next(); c_.vz = next(); c_.divv = next(); c_.p = next();
    c_.df = next(); c_.lap = next();
    for (auto& b : rd_buf_[0]) b = next();
    if constexpr (!kStateCopy<T>)
      for (auto& b : rd_buf_[1]) b = next();
    c_.ldx = next(); c_.ldy = next(); c_.ldz = next();
    c_.sh = next(); c_.dtpsi = next(); c_.tmp = next();
    if constexpr (kStateCopy<T>) c_.tmp64 = dnext();
    else c_.tmp64 = reinterpret_cast<double*>(c_.tmp);
    set_phase(0);
    // every field inside its slab (the counts above are the slabs' sizes)
    layout_ok_ = f == static_cast<T*>(slab_) + size_t(kFields) * n_ && dfp == dslab_ + size_t(kDFields) * n_;
  }

  Field field_ptr(int f) const {
    const size_t t = sizeof(T), d = sizeof(double);
    switch (f) {
      case QUASI_FIELD_PSI: return {c_.psi, d};
      case QUASI_FIELD_RHO: return {c_.rho, d};
      case QUASI_FIELD_VX: return {c_.vx, t};
      case QUASI_FIELD_VY: return {c_.vy, t};
      case QUASI_FIELD_VZ: return {c_.vz, t};
      case QUASI_FIELD_P: return {c_.p, t};
      case QUASI_FIELD_DIVV: return {c_.divv, t};
      case QUASI_FIELD_PSIQ: return {c_.psiq, d};
      case QUASI_FIELD_PSIQ_OLD: return {c_.psiq_old, d};
      case QUASI_FIELD_DTPSI: return {cfg_.variant == QUASI_VARIANT_STB ? c_.dtpsi : nullptr, t};
      case QUASI_FIELD_DF: return {c_.df, t};
      default: return {nullptr, t};
    }
  }

  int capture() {
    for (int ph = 0; ph < kPhases; ++ph) {
      int rc = capture_phase(ph);
      if (rc) return rc;
    }
    set_phase(nloop_);
    return QUASI_OK;
  }

  int capture_phase(int ph) {
    cudaGraph_t graph = nullptr;
    set_phase(ph);
    use_tma();
    if (!cuda_ok(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture"))
      return QUASI_ERR_CUDA;
    cudaError_t e = enqueue_step<T>(c_, tb_, tb64_, nloop_dev_, stream_, stream2_, fork_ev_);
    cudaError_t e2 = cudaStreamEndCapture(stream_, &graph);
    if (!cuda_ok(e, "enqueue step") || !cuda_ok(e2, "end capture")) {
      if (graph) cudaGraphDestroy(graph);
      return QUASI_ERR_CUDA;
    }
    size_t nodes = 0;
    cudaGraphGetNodes(graph, nullptr, &nodes);
    std::vector<cudaGraphNode_t> list(nodes);
    cudaGraphGetNodes(graph, list.data(), &nodes);
    graph_kernels_ = 0;
    for (auto nd : list) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++graph_kernels_;
    }
    e = cudaGraphInstantiate(&graph_exec_[ph], graph, 0);
    if (graph_[ph]) cudaGraphDestroy(graph_[ph]);
    graph_[ph] = graph;   // kept for ensembles that launch members as child graphs
    if (!cuda_ok(e, "graph instantiate")) { graph_exec_[ph] = nullptr; return QUASI_ERR_CUDA; }
    return QUASI_OK;
  }

  quasi_config cfg_;
  Geom g_{};
  size_t n_ = 0;
  bool dev_ok_ = false, have_psi_ = false, initialized_ = false;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  void* slab_ = nullptr;
  double* dslab_ = nullptr;   // the double fields
  tc::Tables4 tc_tables_{};   // split-BF16 form: the folded DCT/DST matrices
  void* tc_owned_ = nullptr;
  bool tc_on_ = false;
  // the autotuner's choices (see autotune())
  struct Tuning {
    bool zwarp[2] = {false, true};
    bool xywarp[2][2] = {{false, false}, {false, false}};   // [axis x, y][float, double]
    int tc_axes = 3;
    bool measured = false;
  } tune_;
  bool layout_ok_ = false;
  double* tabs_ = nullptr;
  int* nloop_dev_ = nullptr;
  double* partial_ = nullptr;
  cudaStream_t stream2_ = nullptr;
  cudaEvent_t fork_ev_[12] = {};
  int* tma_err_ = nullptr;
  int sms_ = 148;
  void* host_stage_ = nullptr;
  DevTwiddles<T> tw_[3];
  DevTwiddles<double> tw64_[3];   // FP32 form: the double transforms' tables
  AxisTables<T> tb_{};
  AxisTables<double> tb64_{};
  StepCtx<T> c_{};
  cudaGraphExec_t graph_exec_[kPhases] = {};
  cudaGraph_t graph_[kPhases] = {};
  double* psiq_buf_[3] = {};
  T* nq_buf_[2] = {};
  double* psi_buf_[2] = {};
  T* rd_buf_[2][3] = {};   // grad rho (x, y, z); the second set in the FP64 form only
  int graph_kernels_ = 0;
  long nloop_ = 0;
};

template <typename T>
EngineBase* make_engine(const quasi_config& cfg, std::string& err) {
  auto* e = new Engine<T>(cfg);
  int rc = e->create();
  if (rc) {
    err = e->err;
    delete e;
    return nullptr;
  }
  return e;
}

}  // namespace quasi
