// The extern "C" boundary declared in include/quasi_gpu.h.
#include <cuda_runtime.h>

#include <new>
#include <string>
#include <vector>

#include "engine.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

bool is_axis_len(int n) {
  switch (n) {
    case 8: case 16: case 32: case 64: case 96: case 128: case 192: case 256: case 512: return true;
    default: return false;
  }
}

int device_check(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(QUASI_ERR_NODEVICE, "no CUDA device available (libquasi_gpu has no CPU fallback)");
  }
  if (device < 0 || device >= count) return fail(QUASI_ERR_INVALID, "device ordinal out of range");
  return QUASI_OK;
}

}  // namespace

namespace quasi {

int set_error(int code, const std::string& msg) { return fail(code, msg); }

std::string validate_config(const quasi_config& c) {
  if (!is_axis_len(c.nx) || !is_axis_len(c.ny) || !is_axis_len(c.nz))
    return "each of nx, ny, nz must be one of 8 16 32 64 96 128 192 256 512";
  if (c.nz % 16 != 0) return "nz must be a multiple of 16";
  if ((long)c.nx * c.ny % 16 != 0) return "nx*ny must be a multiple of 16";
  if (c.variant != QUASI_VARIANT_QUASI && c.variant != QUASI_VARIANT_STB) return "unknown variant";
  if (c.precision != QUASI_PREC_FP64 && c.precision != QUASI_PREC_FP32 && c.precision != QUASI_PREC_BF16X3_TC)
    return "unknown precision";
  if (c.emulate_ranks < 1 || c.nx % c.emulate_ranks != 0) return "emulate_ranks must divide nx";
  if (c.emulate_ranks > 1 && c.emulate_ranks % 2 != 0)
    return "emulate_ranks must be 1 or even (the reference's halo exchanges need an even rank count)";
  if (!(c.dt > 0) || !(c.nu_arg > 0) || !(c.q0 > 0) || c.nw <= 0) return "dt, nu, q0 and nw must be positive";
  return "";
}

}  // namespace quasi

struct quasi_handle {
  quasi::EngineBase* eng;
  quasi_config cfg;
};

extern "C" {

int quasi_abi_version(void) { return QUASI_ABI_VERSION; }

const char* quasi_last_error(void) { return g_err.c_str(); }

int quasi_config_default(quasi_config* c, int variant, int nx, int ny, int nz) {
  if (!c) return fail(QUASI_ERR_INVALID, "null config");
  *c = quasi_config{};
  c->nx = nx; c->ny = ny; c->nz = nz;
  c->variant = variant;
  c->precision = QUASI_PREC_FP64;
  c->emulate_ranks = 1;
  c->device = 0;
  c->alpha = 1.0; c->q0 = 1.0; c->nw = 8;
  c->ep_arg = 675.0;   /* epsilon = -0.675: the one-mode coexistence value */
  c->nu_arg = 1.0;
  c->divv_switch = 200;            /* quasi.cpp:161 */
  c->q_pert = 0.5;                 /* quasi-stb.cpp:157 */
  c->autotune = 1;
  if (variant == QUASI_VARIANT_QUASI) {
    c->gamma = 1.0; c->beta = 2.0;                 /* quasi.cpp:183-184 */
    c->amp = 1.34164; c->rho_0 = 0.005; c->kp = 0.5;  /* quasi.cpp:194-196 */
    c->rho_m = 0.0;                                 /* derived: rho_s / 2 */
    c->dt = 0.001;                                  /* quasi.cpp:203 */
  } else if (variant == QUASI_VARIANT_STB) {
    c->gamma = 3.0; c->beta = 0.4;                  /* quasi-stb.cpp:177-178 */
    c->amp = 0.3464101615; c->rho_0 = 0.1; c->kp = 0.5;
    c->rho_m = 0.5;                                 /* quasi-stb.cpp:197 */
    c->dt = 0.0005;                                 /* quasi-stb.cpp:203 */
  } else {
    return fail(QUASI_ERR_INVALID, "unknown variant");
  }
  return QUASI_OK;
}

int quasi_create(const quasi_config* cfg, quasi_handle** out) {
  if (!cfg || !out) return fail(QUASI_ERR_INVALID, "null argument");
  *out = nullptr;
  std::string why = quasi::validate_config(*cfg);
  if (!why.empty()) return fail(QUASI_ERR_INVALID, why);
  int rc = device_check(cfg->device);
  if (rc) return rc;
  std::string err;
  quasi::EngineBase* e = cfg->precision == QUASI_PREC_FP64 ? quasi::make_engine_f64(*cfg, err)
                                                           : quasi::make_engine_f32(*cfg, err);   // FP32, BF16X3_TC
  if (!e) return fail(err.find("allocation") != std::string::npos ? QUASI_ERR_NOMEM : QUASI_ERR_CUDA, err);
  *out = new (std::nothrow) quasi_handle{e, *cfg};
  if (!*out) {
    delete e;
    return fail(QUASI_ERR_NOMEM, "host allocation failed");
  }
  return QUASI_OK;
}

int quasi_destroy(quasi_handle* h) {
  if (!h) return QUASI_OK;
  delete h->eng;
  delete h;
  return QUASI_OK;
}

#define QUASI_CALL(h, expr)                                     \
  do {                                                          \
    if (!(h)) return fail(QUASI_ERR_INVALID, "null handle");    \
    int rc_ = (expr);                                           \
    if (rc_) return fail(rc_, (h)->eng->err);                   \
    return QUASI_OK;                                            \
  } while (0)

int quasi_set_psi(quasi_handle* h, const double* host_psi) {
  if (!host_psi) return fail(QUASI_ERR_INVALID, "null psi");
  QUASI_CALL(h, h->eng->set_psi(host_psi));
}

int quasi_init(quasi_handle* h) { QUASI_CALL(h, h->eng->init()); }

int quasi_step(quasi_handle* h, int nsteps) { QUASI_CALL(h, h->eng->step(nsteps, nullptr)); }

int quasi_step_async(quasi_handle* h, int nsteps) { QUASI_CALL(h, h->eng->step_async(nsteps)); }

int quasi_synchronize(quasi_handle* h) { QUASI_CALL(h, h->eng->synchronize()); }

int quasi_step_timed(quasi_handle* h, int nsteps, double* device_ms) {
  if (!device_ms) return fail(QUASI_ERR_INVALID, "null device_ms");
  QUASI_CALL(h, h->eng->step(nsteps, device_ms));
}

int quasi_tuning(const quasi_handle* h, int out[4]) {
  if (!h || !out) return fail(QUASI_ERR_INVALID, "null argument");
  h->eng->tuning(out);
  return QUASI_OK;
}

int quasi_step_count(const quasi_handle* h, long* nloop) {
  if (!h || !nloop) return fail(QUASI_ERR_INVALID, "null argument");
  *nloop = h->eng->nloop();
  return QUASI_OK;
}

int quasi_step_kernels(quasi_handle* h, int* launches) {
  if (!launches) return fail(QUASI_ERR_INVALID, "null output");
  QUASI_CALL(h, h->eng->step_kernels(launches));
}

int quasi_time_axis_pass(quasi_handle* h, int axis, int reps, double* avg_ms) {
  if (!avg_ms) return fail(QUASI_ERR_INVALID, "null output");
  QUASI_CALL(h, h->eng->time_axis_pass(axis, reps, avg_ms));
}

int quasi_get_field(quasi_handle* h, int field, double* host_out) {
  if (!host_out) return fail(QUASI_ERR_INVALID, "null output");
  QUASI_CALL(h, h->eng->get_field(field, host_out));
}

int quasi_diagnostics(quasi_handle* h, double out[3]) {
  if (!out) return fail(QUASI_ERR_INVALID, "null output");
  QUASI_CALL(h, h->eng->diagnostics(out));
}

int quasi_growth_rate(quasi_handle* h, double* out) {
  if (!out) return fail(QUASI_ERR_INVALID, "null output");
  QUASI_CALL(h, h->eng->growth_rate(out));
}

int quasi_save(quasi_handle* h, const char* path) {
  if (!path) return fail(QUASI_ERR_INVALID, "null path");
  QUASI_CALL(h, h->eng->save(path));
}

int quasi_load(quasi_handle* h, const char* path) {
  if (!path) return fail(QUASI_ERR_INVALID, "null path");
  QUASI_CALL(h, h->eng->load(path));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ensembles: a vector of owned handles stepped together.
// ---------------------------------------------------------------------------
// The members' step graphs of one rotation phase as child graphs of one
// graph per phase: when every member is at the same phase on the same device,
// a step of the whole ensemble is one graph launch (the members' kernels run
// as independent branches).
struct quasi_ensemble {
  std::vector<quasi_handle*> members;
  cudaStream_t stream = nullptr;
  std::vector<cudaGraphExec_t> exec;   // per phase
  int device = -1;
  ~quasi_ensemble() {
    for (auto& e : exec)
      if (e) cudaGraphExecDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
  // one graph per phase over all members; false if the members do not share
  // a device or a phase count
  cudaError_t build(bool* ok) {
    *ok = false;
    if (members.empty()) return cudaSuccess;
    const int dev = members[0]->eng->device(), ph = members[0]->eng->phases();
    for (auto* h : members)
      if (h->eng->device() != dev || h->eng->phases() != ph) return cudaSuccess;
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return e;
    if (!stream && (e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
    exec.assign(ph, nullptr);
    for (int p = 0; p < ph; ++p) {
      cudaGraph_t g = nullptr;
      if ((e = cudaGraphCreate(&g, 0)) != cudaSuccess) return e;
      for (auto* h : members) {
        cudaGraphNode_t node;
        cudaGraph_t child = h->eng->phase_graph(p);
        if (!child) { cudaGraphDestroy(g); return cudaErrorInvalidValue; }
        if ((e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, child)) != cudaSuccess) {
          cudaGraphDestroy(g);
          return e;
        }
      }
      e = cudaGraphInstantiate(&exec[p], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return e;
    }
    device = dev;
    *ok = true;
    return cudaSuccess;
  }
};

namespace {

int member_fail(size_t m, int rc) {
  return fail(rc, "ensemble member " + std::to_string(m) + ": " + g_err);
}

}  // namespace

extern "C" {

int quasi_ensemble_create(int n, const quasi_config* configs, quasi_ensemble** out) {
  if (!out || !configs || n < 1) return fail(QUASI_ERR_INVALID, "need n >= 1 configs and an output pointer");
  *out = nullptr;
  auto* e = new (std::nothrow) quasi_ensemble;
  if (!e) return fail(QUASI_ERR_NOMEM, "host allocation failed");
  for (int m = 0; m < n; ++m) {
    quasi_handle* h = nullptr;
    int rc = quasi_create(&configs[m], &h);
    if (rc) {
      rc = member_fail(m, rc);
      quasi_ensemble_destroy(e);
      return rc;
    }
    e->members.push_back(h);
  }
  *out = e;
  return QUASI_OK;
}

int quasi_ensemble_size(const quasi_ensemble* e, int* n) {
  if (!e || !n) return fail(QUASI_ERR_INVALID, "null argument");
  *n = int(e->members.size());
  return QUASI_OK;
}

int quasi_ensemble_member(quasi_ensemble* e, int m, quasi_handle** out) {
  if (!e || !out) return fail(QUASI_ERR_INVALID, "null argument");
  if (m < 0 || m >= int(e->members.size())) return fail(QUASI_ERR_INVALID, "member index out of range");
  *out = e->members[m];
  return QUASI_OK;
}

int quasi_ensemble_init(quasi_ensemble* e) {
  if (!e) return fail(QUASI_ERR_INVALID, "null ensemble");
  for (size_t m = 0; m < e->members.size(); ++m) {
    int rc = quasi_init(e->members[m]);
    if (rc) return member_fail(m, rc);
  }
  return QUASI_OK;
}

int quasi_ensemble_step(quasi_ensemble* e, int nsteps) {
  if (!e) return fail(QUASI_ERR_INVALID, "null ensemble");
  if (nsteps < 0) return fail(QUASI_ERR_INVALID, "nsteps < 0");
  // members in lockstep (initialised, same phase): one graph launch per step
  bool lockstep = !e->members.empty();
  const int ph = e->members.empty() ? 1 : e->members[0]->eng->phases();
  const long phase0 = e->members.empty() ? 0 : e->members[0]->eng->nloop() % ph;
  for (auto* h : e->members)
    lockstep = lockstep && h->eng->initialized() && h->eng->phase_graph(0) && h->eng->nloop() % ph == phase0;
  if (lockstep && e->exec.empty()) {
    bool ok = false;
    cudaError_t ce = e->build(&ok);
    if (ce != cudaSuccess) return fail(QUASI_ERR_CUDA, std::string("ensemble graph: ") + cudaGetErrorString(ce));
    lockstep = ok;
  }
  if (lockstep && !e->exec.empty()) {
    cudaSetDevice(e->device);
    for (int s = 0; s < nsteps; ++s) {
      cudaError_t ce = cudaGraphLaunch(e->exec[(phase0 + s) % ph], e->stream);
      if (ce != cudaSuccess) return fail(QUASI_ERR_CUDA, std::string("ensemble graph launch: ") + cudaGetErrorString(ce));
    }
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    for (auto* h : e->members) h->eng->note_steps(nsteps);
    if (ce != cudaSuccess) return fail(QUASI_ERR_CUDA, std::string("ensemble step: ") + cudaGetErrorString(ce));
    for (size_t m = 0; m < e->members.size(); ++m) {   // each member's wait-timeout flag
      int rc = quasi_synchronize(e->members[m]);
      if (rc) return member_fail(m, rc);
    }
    return QUASI_OK;
  }
  // enqueue everything first; then wait for every member (all of them, even
  // after an error, so that no member is left running)
  int first = QUASI_OK;
  std::string first_err;
  size_t enq = 0;
  for (; enq < e->members.size(); ++enq) {
    int rc = quasi_step_async(e->members[enq], nsteps);
    if (rc) {
      first = member_fail(enq, rc);
      first_err = g_err;
      break;
    }
  }
  for (size_t m = 0; m < enq; ++m) {
    int rc = quasi_synchronize(e->members[m]);
    if (rc && first == QUASI_OK) {
      first = member_fail(m, rc);
      first_err = g_err;
    }
  }
  if (first) g_err = first_err;
  return first;
}

int quasi_ensemble_growth_rates(quasi_ensemble* e, double* out) {
  if (!e || !out) return fail(QUASI_ERR_INVALID, "null argument");
  for (size_t m = 0; m < e->members.size(); ++m) {
    int rc = quasi_growth_rate(e->members[m], &out[m]);
    if (rc) return member_fail(m, rc);
  }
  return QUASI_OK;
}

int quasi_ensemble_destroy(quasi_ensemble* e) {
  if (!e) return QUASI_OK;
  for (quasi_handle* h : e->members) quasi_destroy(h);
  delete e;
  return QUASI_OK;
}

}  // extern "C"
