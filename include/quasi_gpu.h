/* libquasi_gpu: the quasi-incompressible smectic-isotropic pseudo-spectral
 * time step of evitral/smaiso-quasi on one NVIDIA B200 (sm_100a).
 *
 * The reference has no library interface: its step lives inside main() of
 * quasi/quasi.cpp (and quasi/quasi-stb.cpp) behind FFTW-MPI's plan/execute
 * calls.  Each entry point below names the reference code it replaces.
 *
 * Conventions
 *   - Every function returns 0 on success and a negative QUASI_ERR_* code on
 *     failure; quasi_last_error() returns a message for the calling thread.
 *   - Host arrays use the reference layout a[(i*ny + j)*nz + k] (z fastest,
 *     x the reference's MPI slab axis), doubles, nx*ny*nz elements.
 *   - The library owns all device memory of a handle.  A handle is
 *     single-threaded and issues its work on its own CUDA stream.
 */
#ifndef QUASI_GPU_H_
#define QUASI_GPU_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QUASI_ABI_VERSION 1

#if defined(__GNUC__)
#define QUASI_API __attribute__((visibility("default")))
#else
#define QUASI_API
#endif

enum quasi_status {
  QUASI_OK = 0,
  QUASI_ERR_INVALID = -1,    /* bad argument or configuration */
  QUASI_ERR_CUDA = -2,       /* a CUDA call failed */
  QUASI_ERR_NOMEM = -3,      /* device or host allocation failed */
  QUASI_ERR_STATE = -4,      /* call out of order (e.g. step before init) */
  QUASI_ERR_IO = -5,         /* checkpoint file missing, short or corrupt */
  QUASI_ERR_NODEVICE = -6,   /* no usable CUDA device */
  QUASI_ERR_UNSUPPORTED = -7,/* valid request this build does not implement */
  QUASI_ERR_TIMEOUT = -8     /* a kernel's bounded wait gave up (a tile copy
                                never completed); the context stays usable */
};

enum quasi_variant {
  QUASI_VARIANT_QUASI = 0, /* quasi/quasi.cpp: density-varying model */
  QUASI_VARIANT_STB = 1    /* quasi/quasi-stb.cpp: pure smectic, Crank-Nicolson */
};

enum quasi_precision {
  QUASI_PREC_FP64 = 0,     /* plain form: every field and transform in double */
  QUASI_PREC_FP32 = 1,     /* fields and transforms in float; in double: the
                              carried state psi^, psi, grad psi, the density
                              chain (law, filter, rho, divv quotient),
                              constants, the update and the reductions */
  QUASI_PREC_BF16X3_TC = 2 /* the FP32 form with its plain x / y transforms of
                              length 256 as split-BF16 (three-product)
                              contractions on the tensor cores, FP32
                              accumulation; r2r plans: x / y on the tensor
                              cores, z by FFT */
};

enum quasi_field {
  QUASI_FIELD_PSI = 0,      /* psi_local          */
  QUASI_FIELD_RHO = 1,      /* rho_local          */
  QUASI_FIELD_VX = 2,       /* velx_local         */
  QUASI_FIELD_VY = 3,       /* vely_local         */
  QUASI_FIELD_VZ = 4,       /* velz_local         */
  QUASI_FIELD_P = 5,        /* p_local            */
  QUASI_FIELD_DIVV = 6,     /* divv_local         */
  QUASI_FIELD_PSIQ = 7,     /* psiq_local (scaled spectral psi) */
  QUASI_FIELD_PSIQ_OLD = 8, /* psiq_old_local     */
  QUASI_FIELD_DTPSI = 9,    /* dtpsi_local (quasi-stb only) */
  QUASI_FIELD_DF = 10,      /* dfDlapPsi_local    */
  QUASI_FIELD_COUNT = 11
};

/* Model and run configuration.  quasi_config_default() fills the reference's
 * compile-time constants (quasi.cpp:155-219 / quasi-stb.cpp:149-220). */
typedef struct quasi_config {
  int nx, ny, nz;       /* grid; each 2^a 3^b in {8..512}, nz % 16 == 0  */
  int variant;          /* enum quasi_variant                            */
  int precision;        /* enum quasi_precision                          */
  int emulate_ranks;    /* reproduce an MPI run of this many ranks (1 or
                           even, dividing nx): quasi.cpp:1641-1690 reads the
                           previous rank's first x plane at rank boundaries */
  int device;           /* CUDA device ordinal                           */
  double nu_arg;        /* argv[1]: nu (quasi) or nu/0.1 (quasi-stb)     */
  double ep_arg;        /* argv[2]: epsilon = -0.001 * ep_arg            */
  double gamma, beta, alpha, q0;
  double amp;           /* Amp: enters rho_s = kp*Amp + rho_0            */
  double rho_0, kp;
  double rho_m;         /* <= 0: rho_s / 2 (quasi.cpp:198)               */
  double dt;
  int nw;               /* points per wavelength: dx = 2 pi / (q0 nw)    */
  int divv_switch;      /* divv on after this step, p coupling one later */
  double q_pert;        /* quasi-stb growth-rate probe wavenumber Q       */
  int autotune;         /* 1 (default): quasi_create times the candidate
                           kernels of each tunable pass (z pass as CTA or
                           warp tiles per type; FFT or tensor-core x / y
                           passes in the BF16X3_TC form) on this grid and
                           keeps the fastest, remembered per grid and
                           device for later handles; 0: fixed defaults;
                           2: every pass as warp tiles where it can be     */
} quasi_config;

typedef struct quasi_handle quasi_handle;

QUASI_API int quasi_abi_version(void);
QUASI_API const char* quasi_last_error(void);

/* Fill `cfg` with the reference defaults of `variant` on an nx*ny*nz grid. */
QUASI_API int quasi_config_default(quasi_config* cfg, int variant, int nx, int ny, int nz);

/* Allocate device state.  Replaces quasi.cpp:228-495 (MPI init, slab
 * decomposition, 39 field vectors, 8 fftw_mpi_plan_r2r_3d plans). */
QUASI_API int quasi_create(const quasi_config* cfg, quasi_handle** out);
QUASI_API int quasi_destroy(quasi_handle* h);

/* Initial psi from host memory (the reference fills psi_local at
 * quasi.cpp:506-589 or reads it at quasi.cpp:692-717). */
QUASI_API int quasi_set_psi(quasi_handle* h, const double* host_psi);

/* Pre-loop projection and first nonlinear term, quasi.cpp:875-951. */
QUASI_API int quasi_init(quasi_handle* h);

/* Advance nsteps steps (the body of the while loop, quasi.cpp:1014-1965);
 * the step is one CUDA graph.  Returns when the steps have completed. */
QUASI_API int quasi_step(quasi_handle* h, int nsteps);

/* As quasi_step, timing the steps with CUDA events on the handle's stream;
 * *device_ms receives the elapsed device time of the nsteps steps. */
QUASI_API int quasi_step_timed(quasi_handle* h, int nsteps, double* device_ms);

/* The autotuner's choices for this handle: out[0] / out[1] = the float /
 * double passes that run as warp tiles (bit 0 z, bit 1 x, bit 2 y; the rest as
 * CTA tiles), out[2] = axes (bit 0 x, bit 1 y) whose plain float passes run on
 * the tensor cores (BF16X3_TC form), out[3] = 1 if the choices were measured
 * (0: defaults).  No reference counterpart. */
QUASI_API int quasi_tuning(const quasi_handle* h, int out[4]);

/* Kernel launches in one step (kernel nodes of the step's CUDA graph; the
 * graph is captured by the first quasi_step).  No reference counterpart. */
QUASI_API int quasi_step_kernels(quasi_handle* h, int* launches);

/* Average device time of one plain in-place axis pass (axis 0 = x, 1 = y,
 * 2 = z) over `reps` back-to-back launches on the handle's stream, timed
 * with CUDA events; operates on a scratch field.  For roofline reporting. */
QUASI_API int quasi_time_axis_pass(quasi_handle* h, int axis, int reps, double* avg_ms);

/* Enqueue nsteps steps on the handle's stream and return at once, so that
 * several handles (an ensemble of instances) run concurrently on one GPU;
 * quasi_synchronize waits for them and reports any device-side error.
 * Every other call of a handle synchronises by itself.  No reference
 * counterpart (the reference runs one instance per MPI job). */
QUASI_API int quasi_step_async(quasi_handle* h, int nsteps);
QUASI_API int quasi_synchronize(quasi_handle* h);

/* Steps taken since quasi_init (the reference's nLoop). */
QUASI_API int quasi_step_count(const quasi_handle* h, long* nloop);

/* Copy one field to host memory (doubles, reference layout). */
QUASI_API int quasi_get_field(quasi_handle* h, int field, double* host_out);

/* L1 = sum|psi - psi_old| / (dt sum|psi|), mass = sum(rho) dx^3,
 * energy = sum rho(-ep psi^2/2 + alpha df^2/2 - beta psi^4/4 + gamma psi^6/6) dx^3,
 * accumulated in double: quasi.cpp:1969-2033.  out[2] is 0 for quasi-stb. */
QUASI_API int quasi_diagnostics(quasi_handle* h, double out[3]);

/* quasi-stb growth rate (psiq - psiq_old)/(dt psiq_old) at the mode
 * (round(Q/Vqz[1]), 0, round(q0/Vqz[1])): quasi-stb.cpp:2149-2157. */
QUASI_API int quasi_growth_rate(quasi_handle* h, double* out);

/* Exact binary checkpoint of the carried state (psiq, psiq_old, Nq_old,
 * rhoq, rho, rho_old, v, divv, divvq, p, df, psi, psi_old, grad psi, grad rho
 * in the FP64 form, the float copies of psiq and rhoq in the FP32 form, nLoop)
 * with a checksum; a file of another grid, variant or precision is rejected.
 * The reference restarts from psi text only (quasi.cpp:692-717);
 * quasi_set_psi + quasi_init reproduce that. */
QUASI_API int quasi_save(quasi_handle* h, const char* path);
QUASI_API int quasi_load(quasi_handle* h, const char* path);

/* ---- diagnostics without allocation --------------------------------------
 * No counterpart in the reference (its reductions are plain host loops).
 * The same FP64 reductions as quasi_diagnostics, for callers that cannot
 * call cudaMalloc (a device whose memory is owned by another component's
 * pool, a real-time host loop that must not synchronise on an allocation):
 * no handle, nothing allocated; the caller passes its own device fields
 * (nx*ny*nz elements of cfg->precision's type, reference layout) and a host
 * array for the 3 results, and may pass a cudaStream_t (NULL: the default
 * stream); the call returns after the results are on the host.  The partial
 * sums live in a fixed __device__ array of 64 KiB that every GPU loading the
 * library keeps until exit, so grids are limited to 2^25 cells (larger ones
 * are rejected).  The first call on a device looks that array up; make it
 * before any stream capture.  Calls that overlap on the GPU race.
 * The call runs on cfg->device (the caller's current device is restored),
 * rejects field pointers that are not device memory of that device
 * (QUASI_ERR_INVALID), and waits for its stream, so it must not be made on
 * a stream that is being captured (QUASI_ERR_STATE).  dt, q0 and nw must be
 * positive.  df may be NULL for the quasi-stb variant (no energy; out[2] = 0). */
QUASI_API int quasi_diagnostics_noalloc(const quasi_config* cfg, const void* psi, const void* psi_old,
                                        const void* rho, const void* df, double out[3], void* stream);

/* ---- seeded initial conditions (host only, no device needed) -----------
 * The reference builds a focal-conic domain (quasi.cpp:543-589) or reads psi
 * from text (quasi.cpp:692-717); the workloads add planar, undulated,
 * displaced-interface and droplet smectic-isotropic interfaces. */
enum quasi_ic_kind {
  QUASI_IC_PLANAR = 0,     /* A(z) cos(q0 z), A = A0/2 (1 - tanh((z - Lz/2)/w)) */
  QUASI_IC_UNDULATED = 1,  /* A(z) cos(q0 z + delta sin(2pi x/Lx) sin(2pi y/Ly)) */
  QUASI_IC_INTERFACE = 2,  /* A(z-h) cos(q0 (z-h)), h = eps_h cos(q_h x)        */
  QUASI_IC_DROPLET = 3,    /* A(r) cos(q0 z), tanh radial envelope, R = radius_frac L */
  QUASI_IC_STB = 4,        /* quasi-stb.cpp:549-550 undulated layers           */
  QUASI_IC_FOCAL_CONIC = 5 /* quasi.cpp:543-589, size aE = bE = fc_size        */
};
typedef struct quasi_ic {
  int kind;
  unsigned long long seed; /* splitmix64 stream seed for the noise           */
  double noise;            /* uniform noise amplitude on psi                 */
  double delta;            /* undulation amplitude                           */
  double eps_h, q_h;       /* interface displacement                         */
  double radius_frac;      /* droplet radius / box length                    */
  double width_wavelengths;/* tanh envelope width w in wavelengths 2 pi/q0   */
  double amp0;             /* <= 0: A0 = sqrt(9 beta / (10 gamma))            */
  double fc_size;          /* focal-conic aE = bE (argv[3])                  */
} quasi_ic;
QUASI_API int quasi_ic_default(quasi_ic* ic, int kind);
QUASI_API int quasi_initial_condition(const quasi_config* cfg, const quasi_ic* ic, double* host_psi);

/* ---- ensembles of independent instances ------------------------------------
 * n members, each an instance with its own grid, variant, precision, device
 * and constants (configs[m]), stepped together: quasi_ensemble_step enqueues
 * nsteps on every member's stream before it waits for any, so the members
 * share the GPU(s).  Members are reached through quasi_ensemble_member (a
 * handle owned by the ensemble: set_psi, get_field, diagnostics, growth rate,
 * save/load; do not destroy it).  No reference counterpart: the reference
 * runs one instance per MPI job (quasi-stb.cpp:2113-2159 is its growth-rate
 * probe). */
typedef struct quasi_ensemble quasi_ensemble;
QUASI_API int quasi_ensemble_create(int n, const quasi_config* configs, quasi_ensemble** out);
QUASI_API int quasi_ensemble_size(const quasi_ensemble* e, int* n);
QUASI_API int quasi_ensemble_member(quasi_ensemble* e, int m, quasi_handle** out);
/* quasi_init of every member (each must have had quasi_set_psi). */
QUASI_API int quasi_ensemble_init(quasi_ensemble* e);
QUASI_API int quasi_ensemble_step(quasi_ensemble* e, int nsteps);
/* quasi_growth_rate of every member into out[0..n-1] (quasi-stb members). */
QUASI_API int quasi_ensemble_growth_rates(quasi_ensemble* e, double* out);
QUASI_API int quasi_ensemble_destroy(quasi_ensemble* e);

/* ---- lower interface: one 3-D r2r transform with FFTW semantics ---------
 * kind[a] per axis (x, y, z): 0 REDFT10, 1 REDFT01, 2 RODFT10, 3 RODFT01,
 * unnormalised, in place.  Replaces fftw_mpi_plan_r2r_3d / fftw_execute
 * (quasi.cpp:449-495 and every fftw_execute of the loop). */
typedef struct quasi_r2r_plan quasi_r2r_plan;
QUASI_API int quasi_r2r_plan_create(int nx, int ny, int nz, const int kind[3], int precision, int device,
                          quasi_r2r_plan** out);
/* data: device pointer to nx*ny*nz elements (double for FP64, float for
 * FP32); stream: a cudaStream_t or NULL for the plan's own stream. */
QUASI_API int quasi_r2r_execute_device(quasi_r2r_plan* p, void* data, void* stream);
/* host doubles in -> host doubles out (may alias); copies included. */
QUASI_API int quasi_r2r_execute_host(quasi_r2r_plan* p, const double* in, double* out);
QUASI_API int quasi_r2r_plan_destroy(quasi_r2r_plan* p);

/* Fault injection for failure-detection tests (no reference counterpart: the
 * reference has no failure detection).  The plan's next execution issues no
 * copy for tile `skip_tile` of each of its TMA passes and gives every tile
 * wait `poll_limit` polls: the wait of that tile runs out, the kernel drains
 * its other copies, flags the error and returns, and the synchronising
 * execution returns QUASI_ERR_TIMEOUT (the output is then undefined).  Only
 * the next execution is affected. */
QUASI_API int quasi_r2r_inject_wait_timeout(quasi_r2r_plan* p, int skip_tile, unsigned poll_limit);

#ifdef __cplusplus
}
#endif

#endif /* QUASI_GPU_H_ */
