// The quasi-incompressible smectic-isotropic time step (quasi.cpp:1014-1965)
// and its stability variant (quasi-stb.cpp:983-1968) as a sequence of fused
// axis passes.  Every pointwise triple loop of the reference becomes the
// loader (first pass) or storer (last pass) of the transform that consumes or
// produces it, so no intermediate array of the reference is materialised
// unless a later stage reads it.
//
// Templated on the storage/transform type T (double: the plain FP64 form;
// float: the FP32 form).  Wavenumbers, spectral constants, the semi-implicit
// update and all reductions are evaluated in double in both forms.
#pragma once
#include <cuda_runtime.h>

#include "r2r_pass.cuh"

namespace quasi {

enum Variant : int { kQuasi = 0, kStb = 1 };

template <typename T>
struct StepCtx {
  Geom g;
  // per-axis wavenumbers, quasi.cpp:397-431 (DST index n carries mode n+1)
  const double *vqx, *vqy, *vqz, *vsx, *vsy, *vsz;
  double ep, alpha, beta, gamma, q0, kp, rho0, rho_s, rho_m, nu, dt, scale;
  int variant, divv_switch, n0;   // n0: planes per emulated MPI rank (quasi.cpp:1641-1690)
  const int* nloop;               // device step counter (the reference's nLoop)
  int store_dtpsi;
  // spectral state (scaled as the reference scales them).  psiq, psiq_old and
  // psiq_new rotate through three buffers and Nq, Nq_old through two (one
  // captured graph per phase of the rotation), so the update writes its
  // result into a buffer nobody reads in that pass.
  T *psiq, *psiq_old, *psiq_new, *Nq, *Nq_old, *rhoq, *divvq, *Sx, *Sy, *Sz;
  // real fields (psi, psi_old and psi_new rotate through two buffers:
  // psi_new is psi_old's buffer)
  T *psi, *psi_old, *psi_new, *rho, *rho_old, *vx, *vy, *vz, *divv, *p, *df, *lap;
  T *gx, *gy, *gz, *rdx, *rdy, *rdz, *ldx, *ldy, *ldz, *sh, *dtpsi, *tmp;
};

__device__ __forceinline__ double sq(double x) { return x * x; }

// Arithmetic type of the elementwise stages: the storage type.  The
// semi-implicit update and the reductions always use double.
template <typename T> using Arith = T;
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }

template <typename T>
__device__ __forceinline__ size_t at(const StepCtx<T>& c, int i, int j, int k) { return lin(c.g, i, j, k); }

template <typename T>
__device__ __forceinline__ double mq2c(const StepCtx<T>& c, int i, int j, int k) {
  return sq(c.vqx[i]) + sq(c.vqy[j]) + sq(c.vqz[k]);   // quasi.cpp:882
}

// ---------------------------------------------------------------------------
// Spectral loaders (first, x-axis pass of inverse transforms)
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Spectral multipliers of the OUTPUT index (i, j, k) for the TMA x passes
// (the loaders above, in the form the TMA pass applies them).
// ---------------------------------------------------------------------------
template <typename T> struct MDf {      // dfDlapPsi, quasi.cpp:1044
  static constexpr bool kActive = true;
  StepCtx<T> c;
  __device__ double operator()(int i, int j, int k) const { return c.alpha * (c.q0 * c.q0 - mq2c(c, i, j, k)); }
};
template <typename T> struct MLap {     // lapRhoDfDlapPsi, quasi.cpp:1046-1047
  static constexpr bool kActive = true;
  StepCtx<T> c;
  __device__ double operator()(int i, int j, int k) const {
    const double q2 = mq2c(c, i, j, k);
    return -q2 * (c.alpha * (c.q0 * c.q0 - q2));
  }
};
template <typename T> struct MSh {      // -aLin, quasi-stb.cpp:1019
  static constexpr bool kActive = true;
  StepCtx<T> c;
  __device__ double operator()(int i, int j, int k) const {
    const double q2 = mq2c(c, i, j, k);
    return -(c.ep - c.alpha * sq(c.q0 * c.q0 - q2));
  }
};
// Shifted gradient along A, quasi.cpp:1120-1186.  The input is read at
// index + 1 along x or y by the TMA box offset (the row past the end reads as
// zero: the reference's zero top DST index); along z the shift is applied
// when storing (StShiftK), so the multiplier uses the output index k - 1.
template <typename T, int A, bool LAP> struct MGrad {
  static constexpr bool kActive = true;
  StepCtx<T> c;
  __device__ double operator()(int i, int j, int k) const {
    if (A == 2 && k == 0) return 0.0;
    const int ko = A == 2 ? k - 1 : k;
    const double vs = A == 0 ? c.vsx[i] : (A == 1 ? c.vsy[j] : c.vsz[ko]);
    if (!LAP) return -vs;
    const double mq = (A == 0 ? sq(c.vsx[i]) : sq(c.vqx[i])) + (A == 1 ? sq(c.vsy[j]) : sq(c.vqy[j])) +
                      (A == 2 ? sq(c.vsz[ko]) : sq(c.vqz[ko]));
    return mq * vs;   // -mq * (-vs)
  }
};
template <typename T> struct StShiftK {   // value of input k lands at k - 1; k = 0 zeroes nz - 1
  Geom g;
  T* dst;
  __device__ void operator()(int i, int j, int k, T v) const {
    if (k == 0) dst[lin(g, i, j, g.nz - 1)] = T(0);
    else dst[lin(g, i, j, k - 1)] = v;
  }
};

// ---------------------------------------------------------------------------
// Real-space loaders (first, z-axis pass of forward transforms)
// ---------------------------------------------------------------------------

template <typename T> struct LdRealField {
  StepCtx<T> c;
  const T* src;
  __device__ T operator()(int i, int j, int k) const { return src[at(c, i, j, k)]; }
};

// ---------------------------------------------------------------------------
// Storers
// ---------------------------------------------------------------------------

// rhoq = scale CT(rho) exp(-1.57^2 q^2 8)                     quasi.cpp:1260-1261
template <typename T> struct StRhoq {
  StepCtx<T> c;
  __device__ void operator()(int i, int j, int k, T v) const {
    const double q2 = mq2c(c, i, j, k);
    c.rhoq[at(c, i, j, k)] = T(c.scale * double(v) * exp(-1.57 * 1.57 * q2 * 8));
  }
};

// ---------------------------------------------------------------------------
// Elementwise stages.  Each reads every input field once, fully coalesced
// (consecutive threads -> consecutive k), computes the terms shared by its
// outputs once, and leaves the transforms around it plain.
// ---------------------------------------------------------------------------
// Iterate rows (i, j) with threads over k: one 32-bit division per row.
#define QUASI_ROWS_BEGIN(g)                                                                       \
  for (int row = blockIdx.x; row < (g).nx * (g).ny; row += gridDim.x) {                           \
    const int i = row / (g).ny, j = row - i * (g).ny;                                             \
    const size_t base = size_t(row) * (g).nz;                                                     \
    for (int k = threadIdx.x; k < (g).nz; k += blockDim.x) {                                      \
      const size_t id = base + k;
#define QUASI_ROWS_END \
  }                    \
  }

// rho = kp sqrt(q0^2 psi^2 + |grad psi|^2) + rho_0   quasi.cpp:1243-1247
template <typename T>
__global__ void __launch_bounds__(256) rho_law_kernel(StepCtx<T> c, size_t n) {
  using A = Arith<T>;
  const A kp = A(c.kp), q02 = A(c.q0 * c.q0), r0 = A(c.rho0);
  for (size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x; id < n; id += size_t(gridDim.x) * blockDim.x) {
    const A ps = c.psi[id], x = c.gx[id], y = c.gy[id], z = c.gz[id];
    c.rho[id] = T(kp * sqrt(q02 * ps * ps + x * x + y * y + z * z) + r0);
  }
}

// divv (after the switch) and rho_old <- rho          quasi.cpp:1273-1289
template <typename T>
__global__ void __launch_bounds__(256) divv_kernel(StepCtx<T> c, size_t n) {
  using A = Arith<T>;
  const bool on = *c.nloop > c.divv_switch;
  const A idt = A(1.0 / c.dt);
  for (size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x; id < n; id += size_t(gridDim.x) * blockDim.x) {
    const A r = c.rho[id];
    if (on) {
      const A ro = c.rho_old[id];
      const A adv = A(c.vx[id]) * A(c.rdx[id]) + A(c.vy[id]) * A(c.rdy[id]) + A(c.vz[id]) * A(c.rdz[id]);
      c.divv[id] = T(-((r - ro) * idt + adv) / (A(0.5) * (r + ro)));
    }
    c.rho_old[id] = T(r);
  }
}

// stress S (quasi.cpp:1305-1317) or mu grad psi (quasi-stb.cpp:1295-1305)
template <typename T>
__global__ void __launch_bounds__(256) stress_kernel(StepCtx<T> c, size_t n) {
  using A = Arith<T>;
  const A beta = A(c.beta), gamma = A(c.gamma);
  for (size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x; id < n; id += size_t(gridDim.x) * blockDim.x) {
    const A gx = c.gx[id], gy = c.gy[id], gz = c.gz[id];
    if (c.variant == kQuasi) {
      const A rho = c.rho[id];
      const A lr = rho * A(c.lap[id]);
      const A rd = rho * A(c.df[id]);
      c.Sx[id] = T(lr * gx - rd * A(c.ldx[id]));
      c.Sy[id] = T(lr * gy - rd * A(c.ldy[id]));
      c.Sz[id] = T(lr * gz - rd * A(c.ldz[id]));
    } else {
      const A ps = c.psi[id];
      const A mu = A(c.sh[id]) - beta * ps * ps * ps + gamma * ps * ps * ps * ps * ps;
      c.Sx[id] = T(mu * gx);
      c.Sy[id] = T(mu * gy);
      c.Sz[id] = T(mu * gz);
    }
  }
}

// Pressure, staggered Stokes projection and scaled divv, from the spectral
// stress: quasi.cpp:1379-1414 (p), 1420-1872 (v), 1888-1894 (divv).  Writes
// p^ -> p, v^ -> vx/vy/vz, scale*divv^ -> divv; the inverse transforms that
// follow run in place on those fields.
template <typename T>
__global__ void __launch_bounds__(256) project_kernel(StepCtx<T> c) {
  using A = Arith<T>;
  const Geom g = c.g;
  const int nz = g.nz;
  const size_t si = size_t(g.ny) * nz;
  const A scale = A(c.scale), nu = A(c.nu), inu = A(1.0 / c.nu);
  for (int row = blockIdx.x; row < g.nx * g.ny; row += gridDim.x) {
    // everything that depends on (i, j) only
    const int i = row / g.ny, j = row - i * g.ny;
    const size_t base = size_t(row) * nz;
    const A qx = A(c.vqx[i]), qy = A(c.vqy[j]);
    const A vsx = A(c.vsx[i]), vsy = A(c.vsy[j]);
    const bool ip = i > 0, jp = j > 0, last_x = i >= g.nx - 1, last_y = j >= g.ny - 1;
    const bool stb = c.variant == kStb;
    // plane "i - 1" as halo #4 delivers it to vely/velz (quasi.cpp:1649)
    const int isrc = (i % c.n0 == 0) ? i - c.n0 : i - 1;
    const size_t bx = size_t(isrc < 0 ? 0 : isrc) * si + size_t(j) * nz;
    const T* Sx = c.Sx;
    const T* Sy = c.Sy;
    const T* Sz = c.Sz;
    const T* Dq = c.divvq;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
      const size_t id = base + k;
      const bool kp = k > 0, klast = k >= nz - 1;
      // every stencil value is loaded unconditionally from a clamped, in-bounds
      // index (so all loads are in flight together) and masked afterwards
      const size_t im = ip ? id - si : id, ipl = last_x ? id : id + si;
      const size_t jm = jp ? id - nz : id, jpl = last_y ? id : id + nz;
      const size_t km = kp ? id - 1 : id, kpl = klast ? id : id + 1;
      const size_t xs = ip ? bx : base - size_t(j) * nz;   // halo source row (i > 0) or this plane's row 0
      const A sxc = Sx[id], syc = Sy[id], szc = Sz[id], dvc = Dq[id];
      const A sx_im = Sx[im], sy_jm = Sy[jm], sz_km = Sz[km];
      const A sy_x = Sy[ipl - (jp ? nz : 0)], sz_x = Sz[ipl - (kp ? 1 : 0)], dq_x = Dq[ipl];
      const A sx_y = Sx[xs + (last_y ? 0 : nz) + k], sz_y = Sz[jpl - (kp ? 1 : 0)], dq_y = Dq[jpl];
      const A sx_z = Sx[xs + (klast ? k : k + 1)], sy_z = Sy[jm + (klast ? 0 : 1)], dq_z = Dq[kpl];
      const A qz = A(c.vqz[k]);
      // p^: divergence of the stress shifted back onto the cosine grid (quasi.cpp:1379-1414)
      {
        const bool on = stb ? (i * j * k > 0) : (i + j + k != 0);
        A pv = A(0);
        if (on) {
          const A sx = ip ? sx_im : A(0), sy = jp ? sy_jm : A(0), sz = kp ? sz_km : A(0);
          A v = -(qx * sx + qy * sy + qz * sz) * rcp(qx * qx + qy * qy + qz * qz);
          if (stb) v += nu * dvc;
          pv = scale * v;
        }
        c.p[id] = T(pv);
      }
      // v^x (i < nx-1): CM1 = scale/(nu mq), CM2 = Vs/mq  (quasi.cpp:889-899, 1522-1633)
      {
        A v = A(0);
        if (!last_x) {
          const A sy = jp ? sy_x : A(0), sz = kp ? sz_x : A(0);
          const A inv = rcp(vsx * vsx + qy * qy + qz * qz);
          const A dot = vsx * sxc + qy * sy + qz * sz;
          v = (scale * inv * inu) * (sxc - (vsx * inv) * dot + nu * vsx * dq_x);
        }
        c.vx[id] = T(v);
      }
      // v^y, v^z (j < ny-1, k < nz-1)  (quasi.cpp:1683-1872)
      A vy = A(0), vz = A(0);
      if (!last_y && !klast) {
        {
          const A sx = ip ? sx_y : A(0), sz = kp ? sz_y : A(0);
          const A inv = rcp(qx * qx + vsy * vsy + qz * qz);
          const A dot = qx * sx + vsy * syc + qz * sz;
          vy = (scale * inv * inu) * (syc - (vsy * inv) * dot + nu * vsy * dq_y);
        }
        {
          const A vsz = A(c.vsz[k]);
          const A sx = ip ? sx_z : A(0), sy = jp ? sy_z : A(0);
          const A inv = rcp(qx * qx + qy * qy + vsz * vsz);
          const A dot = qx * sx + qy * sy + vsz * szc;
          vz = (scale * inv * inu) * (szc - (vsz * inv) * dot + nu * vsz * dq_z);
        }
      }
      c.vy[id] = T(vy);
      c.vz[id] = T(vz);
      if (!stb) c.divv[id] = T(scale * dvc);
    }
  }
}

// Nonlinear term N (quasi.cpp:1905-1929, quasi-stb.cpp:1900-1924) -> Nq
template <typename T>
__global__ void __launch_bounds__(256) nonlinear_kernel(StepCtx<T> c, size_t n) {
  using A = Arith<T>;
  const bool pcoup = *c.nloop > c.divv_switch + 1;
  const A ep = A(c.ep), beta = A(c.beta), gamma = A(c.gamma), cp = A(c.kp / (c.rho_s * c.rho_s));
  for (size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x; id < n; id += size_t(gridDim.x) * blockDim.x) {
    const A ps = c.psi[id];
    const A p3 = ps * ps * ps, p5 = p3 * ps * ps;
    const A adv = A(c.vx[id]) * A(c.gx[id]) + A(c.vy[id]) * A(c.gy[id]) + A(c.vz[id]) * A(c.gz[id]);
    A nv;
    if (c.variant == kQuasi) {
      const A rho = c.rho[id];
      nv = rho * (ep * ps - A(c.df[id]) + beta * p3 - gamma * p5) - rho * A(c.lap[id]) - adv;
      if (pcoup) {
        const A a = c.rdx[id], b = c.rdy[id], d = c.rdz[id];
        nv += A(c.p[id]) * cp * sqrt(a * a + b * b + d * d);
      }
    } else {
      if (c.store_dtpsi) {
        const A mu = A(c.sh[id]) - beta * p3 + gamma * p5;
        c.dtpsi[id] = T(-mu - adv);   // quasi-stb.cpp:1909-1912, rho == 1
      }
      nv = beta * p3 - gamma * p5 - adv;
    }
    c.Nq[id] = T(nv);
  }
}

// Semi-implicit update -> psiq_new (quasi.cpp:1944-1962, quasi-stb.cpp:1946-1958)
template <typename T>
__global__ void __launch_bounds__(256) update_kernel(StepCtx<T> c) {
  const Geom g = c.g;
  const bool first = *c.nloop == 1;
  const double dtd2 = c.dt / 2;
  QUASI_ROWS_BEGIN(g)
    const double q2 = mq2c(c, i, j, k);
    const double alin = c.ep - c.alpha * sq(c.q0 * c.q0 - q2);
    const double pq = c.psiq[id];
    const double nq = c.Nq[id];
    const double nq_old = first ? nq : double(c.Nq_old[id]);   // :1936-1938
    double nv;
    if (c.variant == kQuasi) {
      const double c1 = 2.0 - c.dt * c.rho_m * alin, c2 = 1.5 - c.dt * c.rho_m * alin;   // :886-887
      nv = (c1 * pq - 0.5 * double(c.psiq_old[id]) + dtd2 * c.scale * (3.0 * nq - nq_old)) / c2;
    } else {
      const double c1 = 1.0 + dtd2 * alin, c2 = 1.0 - dtd2 * alin;   // quasi-stb.cpp:855-856
      nv = (c1 * pq + dtd2 * c.scale * (3.0 * nq - nq_old)) / c2;
    }
    c.psiq_new[id] = T(nv);
  QUASI_ROWS_END
}

// ---------------------------------------------------------------------------
// 3-D transforms as three passes
// ---------------------------------------------------------------------------
template <typename T>
struct AxisTables {
  Tables<T> t[3];
};

// Inverse: x pass (loader -> dst), y pass, z pass (storer).
template <typename T, class Load, class Store>
cudaError_t inverse3(const Geom& g, const AxisTables<T>& tb, const int kinds[3], Load ld, T* dst, Store st,
                     cudaStream_t s) {
  cudaError_t e;
  if ((e = launch_pass<T, 0>(g, kinds[0], tb.t[0], ld, StoreField<T>{g, dst}, s)) != cudaSuccess) return e;
  if ((e = launch_pass<T, 1>(g, kinds[1], tb.t[1], LoadField<T>{g, dst}, StoreField<T>{g, dst}, s)) != cudaSuccess)
    return e;
  return launch_pass<T, 2>(g, kinds[2], tb.t[2], LoadField<T>{g, dst}, st, s);
}

// Inverse with a spectral multiplier: x pass on mul * src[shifted] -> dst
// through stx, then plain y and z passes in place.
template <typename T, class Mul, class StX>
cudaError_t inverse3_mul(const Geom& g, const AxisTables<T>& tb, const int kinds[3], const T* src, Mul mul, int di,
                         int dj, StX stx, T* dst, cudaStream_t s) {
  cudaError_t e;
  if ((e = launch_mul_x_pass<T>(g, kinds[0], tb.t[0], src, mul, di, dj, stx, s)) != cudaSuccess) return e;
  if ((e = launch_pass<T, 1>(g, kinds[1], tb.t[1], LoadField<T>{g, dst}, StoreField<T>{g, dst}, s)) != cudaSuccess)
    return e;
  return launch_pass<T, 2>(g, kinds[2], tb.t[2], LoadField<T>{g, dst}, StoreField<T>{g, dst}, s);
}

// Forward: z pass (loader -> dst), y pass, x pass (storer).
template <typename T, class Load, class Store>
cudaError_t forward3(const Geom& g, const AxisTables<T>& tb, const int kinds[3], Load ld, T* dst, Store st,
                     cudaStream_t s) {
  cudaError_t e;
  if ((e = launch_pass<T, 2>(g, kinds[2], tb.t[2], ld, StoreField<T>{g, dst}, s)) != cudaSuccess) return e;
  if ((e = launch_pass<T, 1>(g, kinds[1], tb.t[1], LoadField<T>{g, dst}, StoreField<T>{g, dst}, s)) != cudaSuccess)
    return e;
  return launch_pass<T, 0>(g, kinds[0], tb.t[0], LoadField<T>{g, dst}, st, s);
}

// FFTW kinds per plan (quasi.cpp:449-495), axes (x, y, z)
constexpr int kCT[3] = {E10, E10, E10};
constexpr int kiCT[3] = {E01, E01, E01};
constexpr int kSTx[3] = {O10, E10, E10};
constexpr int kSTy[3] = {E10, O10, E10};
constexpr int kSTz[3] = {E10, E10, O10};
constexpr int kiSTx[3] = {O01, E01, E01};
constexpr int kiSTy[3] = {E01, O01, E01};
constexpr int kiSTz[3] = {E01, E01, O01};

static __global__ void bump_counter_kernel(int* n) { *n += 1; }

#define QUASI_TRY(x)                          \
  do {                                        \
    cudaError_t e_ = (x);                     \
    if (e_ != cudaSuccess) return e_;         \
  } while (0)

constexpr int kEwBlocks = 148 * 8;   // elementwise grid: 8 x 256 threads per SM

// One time step, enqueued on `s` (captured into a CUDA graph by the caller).
template <typename T>
cudaError_t enqueue_step(const StepCtx<T>& c, const AxisTables<T>& tb, int* nloop_dev, cudaStream_t s) {
  const Geom g = c.g;
  const size_t n = size_t(g.nx) * g.ny * g.nz;
  bump_counter_kernel<<<1, 1, 0, s>>>(nloop_dev);
  QUASI_TRY(cudaGetLastError());
  auto st = [&](T* d) { return StoreField<T>{g, d}; };
  auto ld = [&](T* d) { return LoadField<T>{g, d}; };
  if (c.variant == kQuasi) {
    // a3 prologue quasi.cpp:1036-1057
    QUASI_TRY(inverse3_mul(g, tb, kiCT, c.psiq, MDf<T>{c}, 0, 0, st(c.df), c.df, s));
    QUASI_TRY(inverse3_mul(g, tb, kiCT, c.psiq, MLap<T>{c}, 0, 0, st(c.lap), c.lap, s));
    // a4 gradients quasi.cpp:1120-1232
    QUASI_TRY(inverse3_mul(g, tb, kiSTx, c.psiq, MGrad<T, 0, false>{c}, 1, 0, st(c.gx), c.gx, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTy, c.psiq, MGrad<T, 1, false>{c}, 0, 1, st(c.gy), c.gy, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTz, c.psiq, MGrad<T, 2, false>{c}, 0, 0, StShiftK<T>{g, c.gz}, c.gz, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTx, c.rhoq, MGrad<T, 0, false>{c}, 1, 0, st(c.rdx), c.rdx, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTy, c.rhoq, MGrad<T, 1, false>{c}, 0, 1, st(c.rdy), c.rdy, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTz, c.rhoq, MGrad<T, 2, false>{c}, 0, 0, StShiftK<T>{g, c.rdz}, c.rdz, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTx, c.psiq, MGrad<T, 0, true>{c}, 1, 0, st(c.ldx), c.ldx, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTy, c.psiq, MGrad<T, 1, true>{c}, 0, 1, st(c.ldy), c.ldy, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTz, c.psiq, MGrad<T, 2, true>{c}, 0, 0, StShiftK<T>{g, c.ldz}, c.ldz, s));
    // a5 density + filter quasi.cpp:1237-1268 (rho doubles as the scratch)
    rho_law_kernel<T><<<kEwBlocks, 256, 0, s>>>(c, n);
    QUASI_TRY(cudaGetLastError());
    QUASI_TRY(forward3(g, tb, kCT, ld(c.rho), c.rho, StRhoq<T>{c}, s));
    QUASI_TRY(inverse3(g, tb, kiCT, ld(c.rhoq), c.rho, st(c.rho), s));
    // a6 divv quasi.cpp:1273-1293
    divv_kernel<T><<<kEwBlocks, 256, 0, s>>>(c, n);
    QUASI_TRY(cudaGetLastError());
    QUASI_TRY(forward3(g, tb, kCT, ld(c.divv), c.divvq, st(c.divvq), s));
  } else {
    // quasi-stb.cpp:1005-1038 (the unused dRho transform is elided)
    QUASI_TRY(inverse3_mul(g, tb, kiCT, c.psiq, MSh<T>{c}, 0, 0, st(c.sh), c.sh, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTx, c.psiq, MGrad<T, 0, false>{c}, 1, 0, st(c.gx), c.gx, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTy, c.psiq, MGrad<T, 1, false>{c}, 0, 1, st(c.gy), c.gy, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTz, c.psiq, MGrad<T, 2, false>{c}, 0, 0, StShiftK<T>{g, c.gz}, c.gz, s));
    // rho == 1, divv == 0, grad rho == 0 (rhoq never leaves 0): quasi-stb.cpp:1232
  }
  // a7 stress quasi.cpp:1298-1330
  stress_kernel<T><<<kEwBlocks, 256, 0, s>>>(c, n);
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(forward3(g, tb, kSTx, ld(c.Sx), c.Sx, st(c.Sx), s));
  QUASI_TRY(forward3(g, tb, kSTy, ld(c.Sy), c.Sy, st(c.Sy), s));
  QUASI_TRY(forward3(g, tb, kSTz, ld(c.Sz), c.Sz, st(c.Sz), s));
  // a8 pressure, a9 velocity, a10 scaled divv quasi.cpp:1336-1900
  project_kernel<T><<<kEwBlocks, 256, 0, s>>>(c);
  QUASI_TRY(cudaGetLastError());
  if (c.variant == kQuasi) QUASI_TRY(inverse3(g, tb, kiCT, ld(c.p), c.p, st(c.p), s));
  QUASI_TRY(inverse3(g, tb, kiSTx, ld(c.vx), c.vx, st(c.vx), s));
  QUASI_TRY(inverse3(g, tb, kiSTy, ld(c.vy), c.vy, st(c.vy), s));
  QUASI_TRY(inverse3(g, tb, kiSTz, ld(c.vz), c.vz, st(c.vz), s));
  if (c.variant == kQuasi) QUASI_TRY(inverse3(g, tb, kiCT, ld(c.divv), c.divv, st(c.divv), s));
  // a11 nonlinear term quasi.cpp:1905-1939
  nonlinear_kernel<T><<<kEwBlocks, 256, 0, s>>>(c, n);
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(forward3(g, tb, kCT, ld(c.Nq), c.Nq, st(c.Nq), s));
  // a12 update + iCT quasi.cpp:1944-1965
  update_kernel<T><<<kEwBlocks, 256, 0, s>>>(c);
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(inverse3(g, tb, kiCT, ld(c.psiq_new), c.tmp, st(c.psi_new), s));   // psi_old <- psi by rotation
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// a14 pre-loop: psiq = scale CT(psi); psi = iCT(psiq); Nq = CT(beta psi^3 - gamma psi^5)
// quasi.cpp:905-951
// ---------------------------------------------------------------------------
template <typename T> struct LdInitN {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const double ps = c.psi[at(c, i, j, k)];
    return T(c.beta * ps * ps * ps - c.gamma * ps * ps * ps * ps * ps);
  }
};

template <typename T>
__global__ void init_state_kernel(StepCtx<T> c, size_t n) {
  for (size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x; id < n; id += size_t(gridDim.x) * blockDim.x) {
    c.psiq_old[id] = c.psiq[id];   // quasi.cpp:939
    c.psi_old[id] = c.psi[id];   // quasi.cpp:948
    c.divv[id] = T(0);
    c.divvq[id] = T(0);
    c.rhoq[id] = T(0);
    c.rho_old[id] = T(0);
    c.vx[id] = T(0);
    c.vy[id] = T(0);
    c.vz[id] = T(0);
    c.p[id] = T(0);
    c.rho[id] = c.variant == kQuasi ? T(0) : T(1);
  }
}

template <typename T>
cudaError_t enqueue_init(const StepCtx<T>& c, const AxisTables<T>& tb, int* nloop_dev, cudaStream_t s) {
  const Geom g = c.g;
  QUASI_TRY(forward3(g, tb, kCT, LdRealField<T>{c, c.psi}, c.psiq, ScaleStore<T>{g, c.psiq, T(c.scale)}, s));
  QUASI_TRY(inverse3(g, tb, kiCT, LdRealField<T>{c, c.psiq}, c.psi, StoreField<T>{g, c.psi}, s));
  QUASI_TRY(forward3(g, tb, kCT, LdInitN<T>{c}, c.Nq_old, StoreField<T>{g, c.Nq_old}, s));
  const size_t n = size_t(g.nx) * g.ny * g.nz;
  init_state_kernel<T><<<592, 256, 0, s>>>(c, n);
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(cudaMemsetAsync(nloop_dev, 0, sizeof(int), s));
  return cudaSuccess;
}

}  // namespace quasi
