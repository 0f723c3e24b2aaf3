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
  // spectral state (scaled as the reference scales them)
  T *psiq, *psiq_old, *Nq, *Nq_old, *rhoq, *divvq, *Sx, *Sy, *Sz;
  // real fields
  T *psi, *psi_old, *rho, *rho_old, *vx, *vy, *vz, *divv, *p, *df, *lap;
  T *gx, *gy, *gz, *rdx, *rdy, *rdz, *ldx, *ldy, *ldz, *sh, *dtpsi, *tmp;
};

__device__ __forceinline__ double sq(double x) { return x * x; }

template <typename T>
__device__ __forceinline__ size_t at(const StepCtx<T>& c, int i, int j, int k) { return lin(c.g, i, j, k); }

template <typename T>
__device__ __forceinline__ double mq2c(const StepCtx<T>& c, int i, int j, int k) {
  return sq(c.vqx[i]) + sq(c.vqy[j]) + sq(c.vqz[k]);   // quasi.cpp:882
}

// ---------------------------------------------------------------------------
// Spectral loaders (first, x-axis pass of inverse transforms)
// ---------------------------------------------------------------------------

// dfDlapPsi = alpha (q0^2 - q^2) psiq                       quasi.cpp:1044
template <typename T> struct LdDf {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    return T(c.alpha * (c.q0 * c.q0 - mq2c(c, i, j, k)) * double(c.psiq[at(c, i, j, k)]));
  }
};

// lapRhoDfDlapPsi = -q^2 dfDlapPsi                           quasi.cpp:1046-1047
template <typename T> struct LdLap {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const double q2 = mq2c(c, i, j, k);
    const double df = c.alpha * (c.q0 * c.q0 - q2) * double(c.psiq[at(c, i, j, k)]);
    return T(-q2 * df);
  }
};

// sh = -aLin psiq,  aLin = ep - alpha (q0^2 - q^2)^2          quasi-stb.cpp:1019
template <typename T> struct LdSh {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const double q2 = mq2c(c, i, j, k);
    const double alin = c.ep - c.alpha * sq(c.q0 * c.q0 - q2);
    return T(-alin * double(c.psiq[at(c, i, j, k)]));
  }
};

// Shifted spectral gradient along axis A: G[n] = -Vs[n] X[n+1], top index 0
// (quasi.cpp:1120-1164).  LAP = true multiplies by -|q_s|^2 (quasi.cpp:1169-1186).
template <typename T, int A, bool LAP> struct LdGrad {
  StepCtx<T> c;
  const T* src;
  __device__ T operator()(int i, int j, int k) const {
    const int n = A == 0 ? i : (A == 1 ? j : k);
    const int len = A == 0 ? c.g.nx : (A == 1 ? c.g.ny : c.g.nz);
    if (n >= len - 1) return T(0);
    const int i1 = i + (A == 0), j1 = j + (A == 1), k1 = k + (A == 2);
    const double vs = A == 0 ? c.vsx[i] : (A == 1 ? c.vsy[j] : c.vsz[k]);
    const double gval = -vs * double(src[at(c, i1, j1, k1)]);
    if (!LAP) return T(gval);
    const double mq = (A == 0 ? sq(c.vsx[i]) : sq(c.vqx[i])) + (A == 1 ? sq(c.vsy[j]) : sq(c.vqy[j])) +
                      (A == 2 ? sq(c.vsz[k]) : sq(c.vqz[k]));
    return T(-mq * gval);
  }
};

// Pressure from the divergence of the shifted stress  quasi.cpp:1379-1414,
// quasi-stb.cpp:1397-1404 (mask i*j*k > 0 and (4/3)*nu*divv with 4/3 == 1).
template <typename T> struct LdP {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const bool on = c.variant == kQuasi ? (i + j + k != 0) : (i * j * k > 0);
    if (!on) return T(0);
    const double sx = i > 0 ? double(c.Sx[at(c, i - 1, j, k)]) : 0.0;
    const double sy = j > 0 ? double(c.Sy[at(c, i, j - 1, k)]) : 0.0;
    const double sz = k > 0 ? double(c.Sz[at(c, i, j, k - 1)]) : 0.0;
    const double q2 = mq2c(c, i, j, k);
    double v = -(c.vqx[i] * sx + c.vqy[j] * sy + c.vqz[k] * sz) / q2;
    if (c.variant == kStb) v += c.nu * double(c.divvq[at(c, i, j, k)]);
    return T(c.scale * v);
  }
};

// Staggered Stokes projection of the stress, quasi.cpp:1420-1872.
template <typename T> struct LdVx {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    if (i >= c.g.nx - 1) return T(0);   // last global x plane stays 0 (:1522-1548)
    const double sx = double(c.Sx[at(c, i, j, k)]);
    const double sy = j > 0 ? double(c.Sy[at(c, i + 1, j - 1, k)]) : 0.0;
    const double sz = k > 0 ? double(c.Sz[at(c, i + 1, j, k - 1)]) : 0.0;
    const double vs = c.vsx[i];
    const double mq = sq(vs) + sq(c.vqy[j]) + sq(c.vqz[k]);
    const double cm1 = c.scale / (c.nu * mq), cm2 = vs / mq;   // :889-891
    const double dot = vs * sx + c.vqy[j] * sy + c.vqz[k] * sz;
    return T(cm1 * (sx - cm2 * dot + c.nu * vs * double(c.divvq[at(c, i + 1, j, k)])));
  }
};

// Sx at the plane "i-1" as halo #4 delivers it: on emulated rank r >= 1 the
// rank's first plane receives the previous rank's FIRST plane (quasi.cpp:1649).
template <typename T>
__device__ __forceinline__ int halo4_src(const StepCtx<T>& c, int i) {
  return (i % c.n0 == 0) ? i - c.n0 : i - 1;
}

template <typename T> struct LdVy {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    if (j >= c.g.ny - 1 || k >= c.g.nz - 1) return T(0);   // :1684-1685,1728-1730
    const double sx = i > 0 ? double(c.Sx[at(c, halo4_src(c, i), j + 1, k)]) : 0.0;
    const double sy = double(c.Sy[at(c, i, j, k)]);
    const double sz = k > 0 ? double(c.Sz[at(c, i, j + 1, k - 1)]) : 0.0;
    const double vs = c.vsy[j];
    const double mq = sq(c.vqx[i]) + sq(vs) + sq(c.vqz[k]);
    const double cm1 = c.scale / (c.nu * mq), cm2 = vs / mq;   // :893-895
    const double dot = c.vqx[i] * sx + vs * sy + c.vqz[k] * sz;
    return T(cm1 * (sy - cm2 * dot + c.nu * vs * double(c.divvq[at(c, i, j + 1, k)])));
  }
};

template <typename T> struct LdVz {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    if (j >= c.g.ny - 1 || k >= c.g.nz - 1) return T(0);
    const double sx = i > 0 ? double(c.Sx[at(c, halo4_src(c, i), j, k + 1)]) : 0.0;
    const double sy = j > 0 ? double(c.Sy[at(c, i, j - 1, k + 1)]) : 0.0;
    const double sz = double(c.Sz[at(c, i, j, k)]);
    const double vs = c.vsz[k];
    const double mq = sq(c.vqx[i]) + sq(c.vqy[j]) + sq(vs);
    const double cm1 = c.scale / (c.nu * mq), cm2 = vs / mq;   // :897-899
    const double dot = c.vqx[i] * sx + c.vqy[j] * sy + vs * sz;
    return T(cm1 * (sz - cm2 * dot + c.nu * vs * double(c.divvq[at(c, i, j, k + 1)])));
  }
};

// divv = iCT(scale divvq)                                    quasi.cpp:1888-1900
template <typename T> struct LdDivvOut {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const { return T(c.scale * double(c.divvq[at(c, i, j, k)])); }
};

// Semi-implicit update (quasi.cpp:1944-1962, quasi-stb.cpp:1946-1958), with the
// state shuffles psiq_old <- psiq, psiq <- new, Nq_old <- Nq folded in.
template <typename T> struct LdUpdate {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const size_t id = at(c, i, j, k);
    const double q2 = mq2c(c, i, j, k);
    const double alin = c.ep - c.alpha * sq(c.q0 * c.q0 - q2);
    const double pq = double(c.psiq[id]);
    const double nq = double(c.Nq[id]);
    const double nq_old = (*c.nloop == 1) ? nq : double(c.Nq_old[id]);   // :1936-1938
    const double dtd2 = c.dt / 2;
    double nv;
    if (c.variant == kQuasi) {
      const double c1 = 2.0 - c.dt * c.rho_m * alin, c2 = 1.5 - c.dt * c.rho_m * alin;   // :886-887
      nv = (c1 * pq - 0.5 * double(c.psiq_old[id]) + dtd2 * c.scale * (3.0 * nq - nq_old)) / c2;
    } else {
      const double c1 = 1.0 + dtd2 * alin, c2 = 1.0 - dtd2 * alin;   // quasi-stb.cpp:855-856
      nv = (c1 * pq + dtd2 * c.scale * (3.0 * nq - nq_old)) / c2;
    }
    c.psiq_old[id] = T(pq);
    c.psiq[id] = T(nv);
    c.Nq_old[id] = T(nq);
    return T(nv);
  }
};

// ---------------------------------------------------------------------------
// Real-space loaders (first, z-axis pass of forward transforms)
// ---------------------------------------------------------------------------

// rho = kp sqrt(q0^2 psi^2 + |grad psi|^2) + rho_0          quasi.cpp:1243-1247
template <typename T> struct LdRhoRaw {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const size_t id = at(c, i, j, k);
    const double ps = c.psi[id], x = c.gx[id], y = c.gy[id], z = c.gz[id];
    return T(c.kp * sqrt(c.q0 * c.q0 * ps * ps + x * x + y * y + z * z) + c.rho0);
  }
};

// Stress S_a (quasi.cpp:1305-1317) / mu grad psi (quasi-stb.cpp:1295-1305)
template <typename T, int A> struct LdS {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const size_t id = at(c, i, j, k);
    const double g = A == 0 ? c.gx[id] : (A == 1 ? c.gy[id] : c.gz[id]);
    if (c.variant == kQuasi) {
      const double rho = c.rho[id];
      const double lr = rho * double(c.lap[id]);
      const double ld = A == 0 ? c.ldx[id] : (A == 1 ? c.ldy[id] : c.ldz[id]);
      return T(lr * g - rho * double(c.df[id]) * ld);
    }
    const double ps = c.psi[id];
    const double mu = double(c.sh[id]) - c.beta * ps * ps * ps + c.gamma * ps * ps * ps * ps * ps;
    return T(mu * g);   // rho == 1
  }
};

// Nonlinear term N (quasi.cpp:1905-1929, quasi-stb.cpp:1900-1924)
template <typename T> struct LdN {
  StepCtx<T> c;
  __device__ T operator()(int i, int j, int k) const {
    const size_t id = at(c, i, j, k);
    const double ps = c.psi[id];
    const double p3 = ps * ps * ps, p5 = p3 * ps * ps;
    const double adv = double(c.vx[id]) * double(c.gx[id]) + double(c.vy[id]) * double(c.gy[id]) +
                       double(c.vz[id]) * double(c.gz[id]);
    if (c.variant == kQuasi) {
      const double rho = c.rho[id];
      double n = rho * (c.ep * ps - double(c.df[id]) + c.beta * p3 - c.gamma * p5) - rho * double(c.lap[id]) - adv;
      if (*c.nloop > c.divv_switch + 1) {
        const double a = c.rdx[id], b = c.rdy[id], d = c.rdz[id];
        n += double(c.p[id]) * c.kp * sqrt(a * a + b * b + d * d) / (c.rho_s * c.rho_s);
      }
      return T(n);
    }
    if (c.store_dtpsi) {
      const double mu = double(c.sh[id]) - c.beta * p3 + c.gamma * p5;
      c.dtpsi[id] = T(-mu - adv);   // quasi-stb.cpp:1909-1912, rho == 1
    }
    return T(c.beta * p3 - c.gamma * p5 - adv);
  }
};

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

// smoothed rho, divv (after the switch) and rho_old          quasi.cpp:1267-1285
template <typename T> struct StRho {
  StepCtx<T> c;
  __device__ void operator()(int i, int j, int k, T v) const {
    const size_t id = at(c, i, j, k);
    const double r = v;
    if (*c.nloop > c.divv_switch) {
      const double ro = c.rho_old[id];
      const double adv = double(c.vx[id]) * double(c.rdx[id]) + double(c.vy[id]) * double(c.rdy[id]) +
                         double(c.vz[id]) * double(c.rdz[id]);
      c.divv[id] = T(-((r - ro) / c.dt + adv) / (0.5 * (r + ro)));
    }
    c.rho[id] = v;
    c.rho_old[id] = v;
  }
};

// psi_old <- psi, psi <- iCT(psiq')                           quasi.cpp:1961-1965
template <typename T> struct StPsi {
  StepCtx<T> c;
  __device__ void operator()(int i, int j, int k, T v) const {
    const size_t id = at(c, i, j, k);
    c.psi_old[id] = c.psi[id];
    c.psi[id] = v;
  }
};

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

// One time step, enqueued on `s` (captured into a CUDA graph by the caller).
template <typename T>
cudaError_t enqueue_step(const StepCtx<T>& c, const AxisTables<T>& tb, int* nloop_dev, cudaStream_t s) {
  const Geom g = c.g;
  bump_counter_kernel<<<1, 1, 0, s>>>(nloop_dev);
  QUASI_TRY(cudaGetLastError());
  auto st = [&](T* d) { return StoreField<T>{g, d}; };
  if (c.variant == kQuasi) {
    // a3 prologue quasi.cpp:1036-1057
    QUASI_TRY(inverse3(g, tb, kiCT, LdDf<T>{c}, c.df, st(c.df), s));
    QUASI_TRY(inverse3(g, tb, kiCT, LdLap<T>{c}, c.lap, st(c.lap), s));
    // a4 gradients quasi.cpp:1120-1232
    QUASI_TRY(inverse3(g, tb, kiSTx, LdGrad<T, 0, false>{c, c.psiq}, c.gx, st(c.gx), s));
    QUASI_TRY(inverse3(g, tb, kiSTy, LdGrad<T, 1, false>{c, c.psiq}, c.gy, st(c.gy), s));
    QUASI_TRY(inverse3(g, tb, kiSTz, LdGrad<T, 2, false>{c, c.psiq}, c.gz, st(c.gz), s));
    QUASI_TRY(inverse3(g, tb, kiSTx, LdGrad<T, 0, false>{c, c.rhoq}, c.rdx, st(c.rdx), s));
    QUASI_TRY(inverse3(g, tb, kiSTy, LdGrad<T, 1, false>{c, c.rhoq}, c.rdy, st(c.rdy), s));
    QUASI_TRY(inverse3(g, tb, kiSTz, LdGrad<T, 2, false>{c, c.rhoq}, c.rdz, st(c.rdz), s));
    QUASI_TRY(inverse3(g, tb, kiSTx, LdGrad<T, 0, true>{c, c.psiq}, c.ldx, st(c.ldx), s));
    QUASI_TRY(inverse3(g, tb, kiSTy, LdGrad<T, 1, true>{c, c.psiq}, c.ldy, st(c.ldy), s));
    QUASI_TRY(inverse3(g, tb, kiSTz, LdGrad<T, 2, true>{c, c.psiq}, c.ldz, st(c.ldz), s));
    // a5 density + filter quasi.cpp:1237-1268 (rho doubles as the scratch)
    QUASI_TRY(forward3(g, tb, kCT, LdRhoRaw<T>{c}, c.rho, StRhoq<T>{c}, s));
    QUASI_TRY(inverse3(g, tb, kiCT, LdRealField<T>{c, c.rhoq}, c.rho, StRho<T>{c}, s));
    // a6 divv -> spectral quasi.cpp:1290-1293
    QUASI_TRY(forward3(g, tb, kCT, LdRealField<T>{c, c.divv}, c.divvq, st(c.divvq), s));
    // a7 stress quasi.cpp:1298-1330
    QUASI_TRY(forward3(g, tb, kSTx, LdS<T, 0>{c}, c.Sx, st(c.Sx), s));
    QUASI_TRY(forward3(g, tb, kSTy, LdS<T, 1>{c}, c.Sy, st(c.Sy), s));
    QUASI_TRY(forward3(g, tb, kSTz, LdS<T, 2>{c}, c.Sz, st(c.Sz), s));
    // a8 pressure quasi.cpp:1379-1418
    QUASI_TRY(inverse3(g, tb, kiCT, LdP<T>{c}, c.p, st(c.p), s));
  } else {
    // quasi-stb.cpp:1005-1038 (the unused dRho transform is elided)
    QUASI_TRY(inverse3(g, tb, kiCT, LdSh<T>{c}, c.sh, st(c.sh), s));
    QUASI_TRY(inverse3(g, tb, kiSTx, LdGrad<T, 0, false>{c, c.psiq}, c.gx, st(c.gx), s));
    QUASI_TRY(inverse3(g, tb, kiSTy, LdGrad<T, 1, false>{c, c.psiq}, c.gy, st(c.gy), s));
    QUASI_TRY(inverse3(g, tb, kiSTz, LdGrad<T, 2, false>{c, c.psiq}, c.gz, st(c.gz), s));
    // rho == 1, divv == 0, grad rho == 0 (rhoq never leaves 0): quasi-stb.cpp:1232
    QUASI_TRY(forward3(g, tb, kSTx, LdS<T, 0>{c}, c.Sx, st(c.Sx), s));
    QUASI_TRY(forward3(g, tb, kSTy, LdS<T, 1>{c}, c.Sy, st(c.Sy), s));
    QUASI_TRY(forward3(g, tb, kSTz, LdS<T, 2>{c}, c.Sz, st(c.Sz), s));
  }
  // a9 velocity quasi.cpp:1420-1884
  QUASI_TRY(inverse3(g, tb, kiSTx, LdVx<T>{c}, c.vx, st(c.vx), s));
  QUASI_TRY(inverse3(g, tb, kiSTy, LdVy<T>{c}, c.vy, st(c.vy), s));
  QUASI_TRY(inverse3(g, tb, kiSTz, LdVz<T>{c}, c.vz, st(c.vz), s));
  if (c.variant == kQuasi) {
    // a10 divv out quasi.cpp:1888-1900
    QUASI_TRY(inverse3(g, tb, kiCT, LdDivvOut<T>{c}, c.divv, st(c.divv), s));
  }
  // a11 nonlinear term quasi.cpp:1905-1939
  QUASI_TRY(forward3(g, tb, kCT, LdN<T>{c}, c.Nq, st(c.Nq), s));
  // a12 update + iCT quasi.cpp:1944-1965
  QUASI_TRY(inverse3(g, tb, kiCT, LdUpdate<T>{c}, c.tmp, StPsi<T>{c}, s));
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
    c.psiq_old[id] = c.psiq[id];
    c.psi_old[id] = c.psi[id];
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
  QUASI_TRY(forward3(g, tb, kCT, LdInitN<T>{c}, c.Nq, StoreField<T>{g, c.Nq}, s));
  const size_t n = size_t(g.nx) * g.ny * g.nz;
  init_state_kernel<T><<<592, 256, 0, s>>>(c, n);
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(cudaMemsetAsync(nloop_dev, 0, sizeof(int), s));
  return cudaSuccess;
}

}  // namespace quasi
