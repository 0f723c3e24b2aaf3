// The quasi-incompressible smectic-isotropic time step (quasi.cpp:1014-1965)
// and its stability variant (quasi-stb.cpp:983-1968) as a sequence of axis
// passes and elementwise stages.  The spectral multipliers and index shifts
// of the reference's pointwise loops (df, lap, -aLin, the shifted gradients,
// the density filter, the scale factors) are applied by the loader of the
// first pass or the storer of the last pass of the transform they belong to;
// the stages that combine several real-space fields (density law, divv,
// stress, projection, nonlinear term, update) are one elementwise kernel
// each, reading every input once in 16-byte packs.
//
// Templated on the storage/transform type T (double: the plain FP64 form;
// float: the FP32 form).  Wavenumbers, spectral constants, the semi-implicit
// update and all reductions are evaluated in double in both forms, and both
// keep in double what the density is built from: the carried spectral state
// psi^, psi and grad psi (and their transforms), the density law, rho^ with
// its Gaussian filter, rho, rho_old and the divv difference quotient.  The
// quotient (rho - rho_old)/dt (quasi.cpp:1279) amplifies step-to-step
// rounding noise of rho by 1/dt = 1000, and the rounding errors of a float
// transform of psi^ lie next to psi's own spectrum (|q| = q0): the density
// law's demodulation sqrt(q0^2 psi^2 + |grad psi|^2) moves them to the low
// wavenumbers that the Gaussian filter keeps.
#pragma once
#include <cuda_runtime.h>

#include "r2r_pass.cuh"
#include "z_pass.cuh"

namespace quasi {

enum Variant : int { kQuasi = 0, kStb = 1 };

template <typename T>
struct StepCtx {
  Geom g;
  // per-axis wavenumbers, quasi.cpp:397-431 (DST index n carries mode n+1)
  const double *vqx, *vqy, *vqz, *vsx, *vsy, *vsz;
  // the density filter exp(-1.57^2 8 q^2) per axis: exp(-1.57^2 8 vq_a^2)
  const double *fx, *fy, *fz;
  double ep, alpha, beta, gamma, q0, kp, rho0, rho_s, rho_m, nu, dt, scale;
  int variant, divv_switch, n0;   // n0: planes per emulated MPI rank (quasi.cpp:1641-1690)
  const int* nloop;               // device step counter (the reference's nLoop)
  int store_dtpsi;
  // spectral state (scaled as the reference scales them).  psiq, psiq_old and
  // psiq_new rotate through three buffers and Nq, Nq_old through two (one
  // captured graph per phase of the rotation), so the update writes its
  // result into a buffer nobody reads in that pass.  psiq and rhoq are held
  // in double; in the FP32 form psiq_t and rhoq_t are their float copies,
  // which the float transforms read (the update and the density filter write
  // both).  In the FP64 form the copies are the fields themselves.
  double *psiq, *psiq_old, *psiq_new, *rhoq;
  T *psiq_t, *rhoq_t;
  T *Nq, *Nq_old, *divvq, *Sx, *Sy, *Sz;
  // the density and its previous value, psi and grad psi, in double (psi,
  // psi_old and psi_new rotate through two buffers: psi_new is psi_old's
  // buffer); tmp64: the scratch of the double transform of psi
  double *rho, *rho_old, *psi, *psi_old, *psi_new, *gx, *gy, *gz, *tmp64;
  // real fields in the storage type
  T *vx, *vy, *vz, *divv, *p, *df, *lap;
  T *rdx, *rdy, *rdz, *ldx, *ldy, *ldz, *sh, *dtpsi, *tmp;
  // FP64 form: grad rho for the next step, computed from the new rho^ with
  // rho itself (rdx, rdy, rdz and these rotate through two buffers); the FP32
  // form transforms grad rho from its float copy of rho^ at the step start
  T *rdnx, *rdny, *rdnz;
};

// The FP32 form keeps separate float copies of psi^ and rho^.
template <typename T> constexpr bool kStateCopy = !std::is_same<T, double>::value;

__device__ __forceinline__ double sq(double x) { return x * x; }

// Arithmetic type of the elementwise stages: the storage type.  The
// semi-implicit update and the reductions always use double.
template <typename T> using Arith = T;
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
// FP32: the hardware reciprocal (within 2 ulp, below the FP32 storage rounding)
__device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }

template <typename T>
__device__ __forceinline__ size_t at(const StepCtx<T>& c, int i, int j, int k) { return lin(c.g, i, j, k); }

template <typename T>
__device__ __forceinline__ double mq2c(const StepCtx<T>& c, int i, int j, int k) {
  return sq(c.vqx[i]) + sq(c.vqy[j]) + sq(c.vqz[k]);   // quasi.cpp:882
}

// ---------------------------------------------------------------------------
// Spectral multipliers of the OUTPUT index (i, j, k) for the x passes of the
// inverse transforms, in double (the x pass rounds the product once).  The
// spectrum concentrates on the ring |q| = q0, where q0^2 - q^2 cancels.
// ---------------------------------------------------------------------------
// Each multiplier splits into a column part (j, k: fixed for a thread of an
// x-pass tile, computed once per tile) and a row part (i, per element):
// row(i, col(j, k)) == operator()(i, j, k).
// On x passes the row part reads one wavenumber table (the axis-table
// protocol of the pass kernels: from(0, w, cl) == row(i, cl) for w = table[i]).
template <typename T> struct MDf {      // dfDlapPsi, quasi.cpp:1044
  static constexpr bool kActive = true;
  template <int AX> static constexpr bool kTable = AX == 0;
  StepCtx<T> c;
  struct Col { double s; };             // qy^2 + qz^2
  __device__ Col col(int j, int k) const {
    const double y = __ldg(c.vqy + j), z = __ldg(c.vqz + k);
    return {y * y + z * z};
  }
  __device__ static double q2w(double x, const Col& cl) { return x * x + cl.s; }   // quasi.cpp:882
  __device__ double q2(int i, const Col& cl) const { return q2w(__ldg(c.vqx + i), cl); }
  __device__ double from(int, double x, const Col& cl) const { return c.alpha * (c.q0 * c.q0 - q2w(x, cl)); }
  __device__ double row(int i, const Col& cl) const { return from(0, __ldg(c.vqx + i), cl); }
  __device__ double operator()(int i, int j, int k) const { return row(i, col(j, k)); }
  __device__ const double* axis_table(int) const { return c.vqx; }
  __device__ Col col_at(int, int j, int k) const { return col(j, k); }
};
template <typename T> struct MLap {     // lapRhoDfDlapPsi, quasi.cpp:1046-1047
  static constexpr bool kActive = true;
  template <int AX> static constexpr bool kTable = AX == 0;
  StepCtx<T> c;
  using Col = typename MDf<T>::Col;
  __device__ Col col(int j, int k) const { return MDf<T>{c}.col(j, k); }
  __device__ double from(int, double x, const Col& cl) const {
    const double q2 = MDf<T>::q2w(x, cl);
    return -q2 * (c.alpha * (c.q0 * c.q0 - q2));
  }
  __device__ double row(int i, const Col& cl) const { return from(0, __ldg(c.vqx + i), cl); }
  __device__ double operator()(int i, int j, int k) const { return row(i, col(j, k)); }
  __device__ const double* axis_table(int) const { return c.vqx; }
  __device__ Col col_at(int, int j, int k) const { return col(j, k); }
};
template <typename T> struct MSh {      // -aLin, quasi-stb.cpp:1019
  static constexpr bool kActive = true;
  template <int AX> static constexpr bool kTable = AX == 0;
  StepCtx<T> c;
  using Col = typename MDf<T>::Col;
  __device__ Col col(int j, int k) const { return MDf<T>{c}.col(j, k); }
  __device__ double from(int, double x, const Col& cl) const {
    const double d = c.q0 * c.q0 - MDf<T>::q2w(x, cl);
    return -(c.ep - c.alpha * (d * d));
  }
  __device__ double row(int i, const Col& cl) const { return from(0, __ldg(c.vqx + i), cl); }
  __device__ double operator()(int i, int j, int k) const { return row(i, col(j, k)); }
  __device__ const double* axis_table(int) const { return c.vqx; }
  __device__ Col col_at(int, int j, int k) const { return col(j, k); }
};
// Shifted gradient along A, quasi.cpp:1120-1186.  The input is read at
// index + 1 along x or y by the TMA box offset (the row past the end reads as
// zero: the reference's zero top DST index); along z the z pass shifts each
// row by one when it stages it, so the multiplier here uses k - 1.
// -vs_A, or with LAP |q_s|^2 vs_A (the shifted wavenumber on axis A).  Axis
// tables: on x passes the x wavenumber (where the row part depends on i); on
// y passes -vs_y alone (the y gradient's multiplier after a plain x pass).
template <typename T, int A, bool LAP> struct MGrad {
  static constexpr bool kActive = true;
  template <int AX> static constexpr bool kTable = (AX == 0 && (A == 0 || LAP)) || (AX == 1 && A == 1 && !LAP);
  StepCtx<T> c;
  struct Col { double vs, s; bool zero; };   // vs_A (A = 1, 2); the j, k part of |q_s|^2
  __device__ Col col(int j, int k) const {
    Col cl{0.0, 0.0, A == 2 && k == 0};
    const int ko = A == 2 ? (k > 0 ? k - 1 : 0) : k;
    const double y = A == 1 ? __ldg(c.vsy + j) : __ldg(c.vqy + j);
    const double z = A == 2 ? __ldg(c.vsz + ko) : __ldg(c.vqz + ko);
    if (A == 1) cl.vs = y;
    if (A == 2) cl.vs = z;
    cl.s = y * y + z * z;
    return cl;
  }
  // x = the x wavenumber of row i (vs_x for A = 0, else vq_x); on y passes
  // (AX = 1) x = vs_y[j]
  __device__ double from(int ax, double x, const Col& cl) const {
    if (ax == 1) return -x;
    if (A == 2 && cl.zero) return 0.0;
    if (!LAP) return A == 0 ? -x : -cl.vs;
    return (x * x + cl.s) * (A == 0 ? x : cl.vs);   // -mq * (-vs)
  }
  __device__ double row(int i, const Col& cl) const {
    if (!LAP && A != 0) return from(0, 0.0, cl);
    return from(0, __ldg((A == 0 ? c.vsx : c.vqx) + i), cl);
  }
  __device__ double operator()(int i, int j, int k) const { return row(i, col(j, k)); }
  __device__ const double* axis_table(int ax) const { return ax == 1 ? c.vsy : (A == 0 ? c.vsx : c.vqx); }
  __device__ Col col_at(int ax, int outer, int k) const { return ax == 1 ? Col{0.0, 0.0, false} : col(outer, k); }
};

// ---------------------------------------------------------------------------
// Storers
// ---------------------------------------------------------------------------

// rhoq = scale CT(rho) exp(-1.57^2 q^2 8)                     quasi.cpp:1260-1261
// The storer of the last (x) pass of the FP64 transform of rho, the Gaussian
// as the product of its per-axis factors (host tables in double).  The values
// are staged for the pass's TMA store (in both forms).
struct StRhoq {
  Geom g;
  double* rhoq;
  double scale;
  const double *fx, *fy, *fz;
  __device__ double value(int i, int j, int k, double v) const {
    return scale * v * (__ldg(fx + i) * __ldg(fy + j) * __ldg(fz + k));
  }
  __host__ __device__ double* stage_dst() const { return rhoq; }
  __device__ void operator()(int i, int j, int k, double v) const { rhoq[lin(g, i, j, k)] = value(i, j, k, v); }
  __device__ void pair(int i, int j, int k, double a, double b) const {
    double2 v;
    v.x = value(i, j, k, a);
    v.y = value(i, j, k + 1, b);
    *reinterpret_cast<double2*>(rhoq + lin(g, i, j, k)) = v;
  }
};
// The FP32 form's storer also writes the float copy that the grad rho
// transforms read: rho^ itself is staged and leaves by the tile's TMA store,
// the copy by plain stores from value().
template <typename T>
struct StRhoqCopy {
  StRhoq r;
  T* rhoq_t;
  __host__ __device__ double* stage_dst() const { return r.rhoq; }
  __device__ double value(int i, int j, int k, double v) const {
    const double x = r.value(i, j, k, v);
    rhoq_t[lin(r.g, i, j, k)] = T(x);
    return x;
  }
  __device__ void operator()(int i, int j, int k, double v) const {
    const double x = r.value(i, j, k, v);
    const size_t id = lin(r.g, i, j, k);
    r.rhoq[id] = x;
    rhoq_t[id] = T(x);
  }
  __device__ void pair(int i, int j, int k, double a, double b) const {
    double2 v;
    v.x = r.value(i, j, k, a);
    v.y = r.value(i, j, k + 1, b);
    const size_t id = lin(r.g, i, j, k);
    *reinterpret_cast<double2*>(r.rhoq + id) = v;
    typename Vec2<T>::type w;
    w.x = T(v.x);
    w.y = T(v.y);
    *reinterpret_cast<typename Vec2<T>::type*>(rhoq_t + id) = w;
  }
};

// ---------------------------------------------------------------------------
// Elementwise stages.  Each reads every input field once, fully coalesced
// (consecutive threads -> consecutive k), computes the terms shared by its
// outputs once, and leaves the transforms around it plain.
// ---------------------------------------------------------------------------
// Elementwise stages move 16 bytes per field access: a Pack is V = 16 /
// sizeof(T) consecutive elements of one row (nz is a multiple of 8, so packs
// never straddle rows).  The flat stages walk packs with a grid-stride loop.
template <typename T>
struct alignas(16) Pack {
  static constexpr int V = 16 / sizeof(T);
  T v[V];
};
template <typename T>
__device__ __forceinline__ Pack<T> ldp(const T* p, size_t pi) {
  Pack<T> r;
  *reinterpret_cast<typename Vec4<T>::type*>(r.v) = reinterpret_cast<const typename Vec4<T>::type*>(p)[pi];
  return r;
}
template <typename T>
__device__ __forceinline__ void stp(T* p, size_t pi, const Pack<T>& r) {
  reinterpret_cast<typename Vec4<T>::type*>(p)[pi] = *reinterpret_cast<const typename Vec4<T>::type*>(r.v);
}
// The double fields beside a pack of V = 16/sizeof(T) elements of a T field:
// the same V elements, in 16-byte loads and stores.
template <int V>
struct DPack {
  double v[V];
};
template <int V>
__device__ __forceinline__ DPack<V> ldd(const double* p, size_t pi) {
  DPack<V> r;
#pragma unroll
  for (int q = 0; q < V / 2; ++q)
    *reinterpret_cast<double2*>(r.v + 2 * q) = reinterpret_cast<const double2*>(p + pi * V)[q];
  return r;
}
template <int V>
__device__ __forceinline__ void std_(double* p, size_t pi, const DPack<V>& r) {
#pragma unroll
  for (int q = 0; q < V / 2; ++q)
    reinterpret_cast<double2*>(p + pi * V)[q] = *reinterpret_cast<const double2*>(r.v + 2 * q);
}
#define QUASI_PACKS(n)                                                                                   \
  for (size_t pi = blockIdx.x * size_t(blockDim.x) + threadIdx.x; pi < (n) / Pack<T>::V;               \
       pi += size_t(gridDim.x) * blockDim.x)

// rho = kp sqrt(q0^2 psi^2 + |grad psi|^2) + rho_0   quasi.cpp:1243-1247
// (in double, into the double scratch of the FP64 transform that follows)
template <typename T>
__global__ void __launch_bounds__(256) rho_law_kernel(StepCtx<T> c, size_t n) {
  constexpr int V = Pack<T>::V;
  const double kp = c.kp, q02 = c.q0 * c.q0, r0 = c.rho0;
  QUASI_PACKS(n) {
    const DPack<V> ps = ldd<V>(c.psi, pi), x = ldd<V>(c.gx, pi), y = ldd<V>(c.gy, pi), z = ldd<V>(c.gz, pi);
    DPack<V> r;
#pragma unroll
    for (int u = 0; u < V; ++u) {
      const double p = ps.v[u], a = x.v[u], b = y.v[u], d = z.v[u];
      r.v[u] = kp * sqrt(q02 * p * p + a * a + b * b + d * d) + r0;
    }
    std_(c.rho, pi, r);
  }
}

// divv (after the switch) and rho_old <- rho          quasi.cpp:1273-1289
// The difference quotient in double from the double rho and rho_old; the
// advection term v . grad rho from the storage-type fields.
template <typename T>
__global__ void __launch_bounds__(256) divv_kernel(StepCtx<T> c, size_t n) {
  constexpr int V = Pack<T>::V;
  const bool on = *c.nloop > c.divv_switch;
  const double idt = 1.0 / c.dt;
  QUASI_PACKS(n) {
    const DPack<V> r = ldd<V>(c.rho, pi);
    if (on) {
      const DPack<V> ro = ldd<V>(c.rho_old, pi);
      const Pack<T> vx = ldp(c.vx, pi), vy = ldp(c.vy, pi), vz = ldp(c.vz, pi);
      const Pack<T> ax = ldp(c.rdx, pi), ay = ldp(c.rdy, pi), az = ldp(c.rdz, pi);
      Pack<T> dv;
#pragma unroll
      for (int u = 0; u < V; ++u) {
        const double rr = r.v[u], o = ro.v[u];
        const double adv = double(vx.v[u]) * double(ax.v[u]) + double(vy.v[u]) * double(ay.v[u]) +
                           double(vz.v[u]) * double(az.v[u]);
        dv.v[u] = T(-((rr - o) * idt + adv) / (0.5 * (rr + o)));
      }
      stp(c.divv, pi, dv);
    }
    std_(c.rho_old, pi, r);
  }
}

// stress S (quasi.cpp:1305-1317) or mu grad psi (quasi-stb.cpp:1295-1305)
template <typename T>
__global__ void __launch_bounds__(256) stress_kernel(StepCtx<T> c, size_t n) {
  using A = Arith<T>;
  constexpr int V = Pack<T>::V;
  const A beta = A(c.beta), gamma = A(c.gamma);
  QUASI_PACKS(n) {
    const DPack<V> gx = ldd<V>(c.gx, pi), gy = ldd<V>(c.gy, pi), gz = ldd<V>(c.gz, pi);
    Pack<T> sx, sy, sz;
    if (c.variant == kQuasi) {
      const DPack<V> rho = ldd<V>(c.rho, pi);
      const Pack<T> lap = ldp(c.lap, pi), df = ldp(c.df, pi);
      const Pack<T> lx = ldp(c.ldx, pi), ly = ldp(c.ldy, pi), lz = ldp(c.ldz, pi);
#pragma unroll
      for (int u = 0; u < V; ++u) {
        const A lr = A(rho.v[u]) * A(lap.v[u]);
        const A rd = A(rho.v[u]) * A(df.v[u]);
        sx.v[u] = T(lr * A(gx.v[u]) - rd * A(lx.v[u]));
        sy.v[u] = T(lr * A(gy.v[u]) - rd * A(ly.v[u]));
        sz.v[u] = T(lr * A(gz.v[u]) - rd * A(lz.v[u]));
      }
    } else {
      const DPack<V> psi = ldd<V>(c.psi, pi);
      const Pack<T> sh = ldp(c.sh, pi);
#pragma unroll
      for (int u = 0; u < V; ++u) {
        const A ps = A(psi.v[u]);
        const A mu = A(sh.v[u]) - beta * ps * ps * ps + gamma * ps * ps * ps * ps * ps;
        sx.v[u] = T(mu * A(gx.v[u]));
        sy.v[u] = T(mu * A(gy.v[u]));
        sz.v[u] = T(mu * A(gz.v[u]));
      }
    }
    stp(c.Sx, pi, sx);
    stp(c.Sy, pi, sy);
    stp(c.Sz, pi, sz);
  }
}

// Pressure, staggered Stokes projection and scaled divv, from the spectral
// stress: quasi.cpp:1379-1414 (p), 1420-1872 (v), 1888-1894 (divv).  Writes
// p^ -> p, v^ -> vx/vy/vz, scale*divv^ -> divv; the inverse transforms that
// follow run in place on those fields.
//
// Blocks are (nz / V) x rows (a multiple of 32 threads): thread x owns the
// pack k = V x .. V x + V - 1 of its row.  Every neighbour row (i +- 1,
// j +- 1, the halo source plane) is read as whole packs; the k - 1 / k + 1
// neighbours come from the adjacent lane's pack by a shuffle, or by one
// scalar load at a warp edge.  Lanes whose neighbour value would cross a row
// end are exactly the masked ones (k = 0 or k = nz - 1).
template <typename T>
__device__ __forceinline__ void shift_prev(const Pack<T>& a, const T* row_ptr, int k0, int lane, bool edge,
                                           T out[Pack<T>::V]) {
  constexpr int V = Pack<T>::V;
  T prev = __shfl_up_sync(0xffffffffu, a.v[V - 1], 1);
  if (edge && k0 > 0) prev = row_ptr[k0 - 1];
  out[0] = prev;
#pragma unroll
  for (int u = 1; u < V; ++u) out[u] = a.v[u - 1];
  (void)lane;
}
template <typename T>
__device__ __forceinline__ void shift_next(const Pack<T>& a, const T* row_ptr, int k0, int nz, bool edge,
                                           T out[Pack<T>::V]) {
  constexpr int V = Pack<T>::V;
  T next = __shfl_down_sync(0xffffffffu, a.v[0], 1);
  if (edge && k0 + V < nz) next = row_ptr[k0 + V];
#pragma unroll
  for (int u = 0; u < V - 1; ++u) out[u] = a.v[u + 1];
  out[V - 1] = next;
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) project_kernel(StepCtx<T> c) {
  using A = Arith<T>;
  constexpr int V = Pack<T>::V;
  const Geom g = c.g;
  const int nz = g.nz, nrows = g.nx * g.ny;
  const size_t ppr = nz / V;   // packs per row
  const int k0 = threadIdx.x * V;
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  const bool first_lane = lane == 0, last_lane = lane == 31;
  const A scale = A(c.scale), nu = A(c.nu), inu = A(1.0 / c.nu);
  const bool stb = c.variant == kStb;
  A qz[V], vsz[V];
#pragma unroll
  for (int u = 0; u < V; ++u) {
    qz[u] = A(c.vqz[k0 + u]);
    vsz[u] = A(c.vsz[k0 + u]);
  }
  const T* Sx = c.Sx;
  const T* Sy = c.Sy;
  const T* Sz = c.Sz;
  const T* Dq = c.divvq;
  for (int rbase = blockIdx.x * blockDim.y; rbase < nrows; rbase += gridDim.x * blockDim.y) {
    const int row0 = rbase + threadIdx.y;
    const bool valid = row0 < nrows;   // uniform loop: every lane reaches the shuffles
    const int row = valid ? row0 : nrows - 1;
    const int i = row / g.ny, j = row - i * g.ny;
    const A qx = A(c.vqx[i]), qy = A(c.vqy[j]);
    const A vsx = A(c.vsx[i]), vsy = A(c.vsy[j]);
    const bool ip = i > 0, jp = j > 0, last_x = i >= g.nx - 1, last_y = j >= g.ny - 1;
    // neighbour rows, clamped in range (their values are masked where clamped)
    const int r_im = ip ? row - g.ny : row;                    // (i-1, j)
    const int r_jm = jp ? row - 1 : row;                       // (i, j-1)
    const int r_ip = last_x ? row : row + g.ny;                // (i+1, j)
    const int r_ipjm = r_ip - (jp ? 1 : 0);                    // (i+1, j-1)
    const int r_jp = last_y ? row : row + 1;                   // (i, j+1)
    // plane "i - 1" as halo #4 delivers it to vely/velz (quasi.cpp:1649)
    const int isrc = (i % c.n0 == 0) ? i - c.n0 : i - 1;
    const int r_xs = ip ? (isrc < 0 ? 0 : isrc) * g.ny + j : i * g.ny;   // halo source row, or this plane's row 0
    const int r_xsy = r_xs + (last_y ? 0 : 1);
    auto P = [&](const T* f, int r) { return ldp(f, size_t(r) * ppr + threadIdx.x); };
    const Pack<T> sxc = P(Sx, row), syc = P(Sy, row), szc = P(Sz, row), dvc = P(Dq, row);
    const Pack<T> sx_im = P(Sx, r_im), sy_jm = P(Sy, r_jm);
    const Pack<T> sy_x = P(Sy, r_ipjm), szx = P(Sz, r_ip), dq_x = P(Dq, r_ip);
    const Pack<T> sx_y = P(Sx, r_xsy), szy = P(Sz, r_jp), dq_y = P(Dq, r_jp);
    const Pack<T> sxs = P(Sx, r_xs);
    // k - 1 neighbours: Sz(i,j), Sz(i+1,j), Sz(i,j+1); k + 1: Sx(src,j), Sy(i,j-1), Dq(i,j)
    T sz_km[V], sz_x[V], sz_y[V], sx_z[V], sy_z[V], dq_z[V];
    shift_prev(szc, Sz + size_t(row) * nz, k0, lane, first_lane, sz_km);
    shift_prev(szx, Sz + size_t(r_ip) * nz, k0, lane, first_lane, sz_x);
    shift_prev(szy, Sz + size_t(r_jp) * nz, k0, lane, first_lane, sz_y);
    shift_next(sxs, Sx + size_t(r_xs) * nz, k0, nz, last_lane, sx_z);
    shift_next(sy_jm, Sy + size_t(r_jm) * nz, k0, nz, last_lane, sy_z);
    shift_next(dvc, Dq + size_t(row) * nz, k0, nz, last_lane, dq_z);
    Pack<T> op, ovx, ovy, ovz, odv;
#pragma unroll
    for (int u = 0; u < V; ++u) {
      const int k = k0 + u;
      const bool kp = k > 0, klast = k >= nz - 1;
      // p^: divergence of the stress shifted back onto the cosine grid (quasi.cpp:1379-1414)
      {
        const bool on = stb ? (i * j * k > 0) : (i + j + k != 0);
        A pv = A(0);
        if (on) {
          const A sx = ip ? A(sx_im.v[u]) : A(0), sy = jp ? A(sy_jm.v[u]) : A(0), sz = kp ? A(sz_km[u]) : A(0);
          A v = -(qx * sx + qy * sy + qz[u] * sz) * rcp(qx * qx + qy * qy + qz[u] * qz[u]);
          if (stb) v += nu * A(dvc.v[u]);
          pv = scale * v;
        }
        op.v[u] = T(pv);
      }
      // v^x (i < nx-1): CM1 = scale/(nu mq), CM2 = Vs/mq  (quasi.cpp:889-899, 1522-1633)
      {
        A v = A(0);
        if (!last_x) {
          const A s0 = sxc.v[u];
          const A sy = jp ? A(sy_x.v[u]) : A(0), sz = kp ? A(sz_x[u]) : A(0);
          const A inv = rcp(vsx * vsx + qy * qy + qz[u] * qz[u]);
          const A dot = vsx * s0 + qy * sy + qz[u] * sz;
          v = (scale * inv * inu) * (s0 - (vsx * inv) * dot + nu * vsx * A(dq_x.v[u]));
        }
        ovx.v[u] = T(v);
      }
      // v^y, v^z (j < ny-1, k < nz-1)  (quasi.cpp:1683-1872)
      A vy = A(0), vz = A(0);
      if (!last_y && !klast) {
        {
          const A s0 = syc.v[u];
          const A sx = ip ? A(sx_y.v[u]) : A(0), sz = kp ? A(sz_y[u]) : A(0);
          const A inv = rcp(qx * qx + vsy * vsy + qz[u] * qz[u]);
          const A dot = qx * sx + vsy * s0 + qz[u] * sz;
          vy = (scale * inv * inu) * (s0 - (vsy * inv) * dot + nu * vsy * A(dq_y.v[u]));
        }
        {
          const A s0 = szc.v[u];
          const A sx = ip ? A(sx_z[u]) : A(0), sy = jp ? A(sy_z[u]) : A(0);
          const A inv = rcp(qx * qx + qy * qy + vsz[u] * vsz[u]);
          const A dot = qx * sx + qy * sy + vsz[u] * s0;
          vz = (scale * inv * inu) * (s0 - (vsz[u] * inv) * dot + nu * vsz[u] * A(dq_z[u]));
        }
      }
      ovy.v[u] = T(vy);
      ovz.v[u] = T(vz);
      odv.v[u] = T(scale * A(dvc.v[u]));
    }
    if (valid) {
      const size_t pi = size_t(row) * ppr + threadIdx.x;
      stp(c.p, pi, op);
      stp(c.vx, pi, ovx);
      stp(c.vy, pi, ovy);
      stp(c.vz, pi, ovz);
      if (!stb) stp(c.divv, pi, odv);
    }
  }
}

// Nonlinear term N (quasi.cpp:1905-1929, quasi-stb.cpp:1900-1924) -> Nq
template <typename T>
__global__ void __launch_bounds__(256) nonlinear_kernel(StepCtx<T> c, size_t n) {
  using A = Arith<T>;
  constexpr int V = Pack<T>::V;
  const bool pcoup = *c.nloop > c.divv_switch + 1;
  const A ep = A(c.ep), beta = A(c.beta), gamma = A(c.gamma), cp = A(c.kp / (c.rho_s * c.rho_s));
  QUASI_PACKS(n) {
    const DPack<V> psi = ldd<V>(c.psi, pi);
    const Pack<T> vx = ldp(c.vx, pi), vy = ldp(c.vy, pi), vz = ldp(c.vz, pi);
    const DPack<V> gx = ldd<V>(c.gx, pi), gy = ldd<V>(c.gy, pi), gz = ldd<V>(c.gz, pi);
    A adv[V], p3[V], p5[V];
#pragma unroll
    for (int u = 0; u < V; ++u) {
      const A ps = A(psi.v[u]);
      p3[u] = ps * ps * ps;
      p5[u] = p3[u] * ps * ps;
      adv[u] = A(vx.v[u]) * A(gx.v[u]) + A(vy.v[u]) * A(gy.v[u]) + A(vz.v[u]) * A(gz.v[u]);
    }
    Pack<T> out;
    if (c.variant == kQuasi) {
      const DPack<V> rho = ldd<V>(c.rho, pi);
      const Pack<T> df = ldp(c.df, pi), lap = ldp(c.lap, pi);
#pragma unroll
      for (int u = 0; u < V; ++u) {
        const A r = A(rho.v[u]), ps = A(psi.v[u]);
        out.v[u] = T(r * (ep * ps - A(df.v[u]) + beta * p3[u] - gamma * p5[u]) - r * A(lap.v[u]) - adv[u]);
      }
      if (pcoup) {
        const Pack<T> a = ldp(c.rdx, pi), b = ldp(c.rdy, pi), d = ldp(c.rdz, pi), p = ldp(c.p, pi);
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const A x = a.v[u], y = b.v[u], z = d.v[u];
          out.v[u] = T(A(out.v[u]) + A(p.v[u]) * cp * sqrt(x * x + y * y + z * z));
        }
      }
    } else {
      if (c.store_dtpsi) {
        const Pack<T> sh = ldp(c.sh, pi);
        Pack<T> dt;
#pragma unroll
        for (int u = 0; u < V; ++u) dt.v[u] = T(-(A(sh.v[u]) - beta * p3[u] + gamma * p5[u]) - adv[u]);   // quasi-stb.cpp:1909-1912, rho == 1
        stp(c.dtpsi, pi, dt);
      }
#pragma unroll
      for (int u = 0; u < V; ++u) out.v[u] = T(beta * p3[u] - gamma * p5[u] - adv[u]);
    }
    stp(c.Nq, pi, out);
  }
}

// Semi-implicit update -> psiq_new (quasi.cpp:1944-1962, quasi-stb.cpp:1946-1958).
// Blocks are (nz / V) x rows: thread x owns the pack at k = V x of row
// blockIdx.x * blockDim.y + y (then + gridDim.x * blockDim.y ...).
template <typename T>
__global__ void __launch_bounds__(256) update_kernel(StepCtx<T> c) {
  constexpr int V = Pack<T>::V;
  const Geom g = c.g;
  const bool first = *c.nloop == 1;
  const double dtd2 = c.dt / 2, dsc = dtd2 * c.scale;
  const int k0 = threadIdx.x * V;
  double qz2[V];
#pragma unroll
  for (int u = 0; u < V; ++u) qz2[u] = sq(c.vqz[k0 + u]);
  const size_t ppr = g.nz / V;   // packs per row
  for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < g.nx * g.ny; row += gridDim.x * blockDim.y) {
    const int i = row / g.ny, j = row - i * g.ny;
    const double qxy = sq(c.vqx[i]) + sq(c.vqy[j]);
    const size_t pi = size_t(row) * ppr + threadIdx.x;
    const DPack<V> pq = ldd<V>(c.psiq, pi);
    const Pack<T> nq = ldp(c.Nq, pi);
    const Pack<T> nqo = first ? nq : ldp(c.Nq_old, pi);   // :1936-1938
    DPack<V> pqo;
    if (c.variant == kQuasi) pqo = ldd<V>(c.psiq_old, pi);
    DPack<V> out;
#pragma unroll
    for (int u = 0; u < V; ++u) {
      const double q2 = qxy + qz2[u];
      const double alin = c.ep - c.alpha * sq(c.q0 * c.q0 - q2);
      const double forcing = dsc * (3.0 * double(nq.v[u]) - double(nqo.v[u]));
      double nv;
      if (c.variant == kQuasi) {
        const double c1 = 2.0 - c.dt * c.rho_m * alin, c2 = 1.5 - c.dt * c.rho_m * alin;   // :886-887
        nv = (c1 * double(pq.v[u]) - 0.5 * double(pqo.v[u]) + forcing) / c2;
      } else {
        const double c1 = 1.0 + dtd2 * alin, c2 = 1.0 - dtd2 * alin;   // quasi-stb.cpp:855-856
        nv = (c1 * double(pq.v[u]) + forcing) / c2;
      }
      out.v[u] = nv;
    }
    std_(c.psiq_new, pi, out);
    if constexpr (kStateCopy<T>) {   // the float copy the next step's transforms read
      Pack<T> t;
#pragma unroll
      for (int u = 0; u < V; ++u) t.v[u] = T(out.v[u]);
      stp(c.psiq_t, pi, t);
    }
  }
}

// ---------------------------------------------------------------------------
// 3-D transforms as three passes
// ---------------------------------------------------------------------------
template <typename T>
struct AxisTables {
  Tables<T> t[3];
};

// y and z passes of `src` (plain field) into `st` (the y pass in place, the
// z pass into st.dst).  kshift = 1: the z pass transforms row[k + 1] (zero at
// the top) in place of row[k], the z shift of a z gradient
// (quasi.cpp:1163-1186).
template <typename T, class Store>
cudaError_t yz3(const Geom& g, const AxisTables<T>& tb, const int kinds[3], T* src, Store st, cudaStream_t s,
                int kshift = 0) {
  cudaError_t e;
  if ((e = launch_pass<T, 1>(g, kinds[1], tb.t[1], LoadField<T>{g, src}, StoreField<T>{g, src}, s)) != cudaSuccess)
    return e;
  if constexpr (IsStoreField<Store>::value) {
    e = launch_zpass<T>(g, kinds[2], tb.t[2], src, st.dst, s, kshift);
    if (e != cudaErrorNotSupported) return e;
  }
  return launch_pass<T, 2>(g, kinds[2], tb.t[2], LoadField<T>{g, src}, st, s, kshift);
}

// Inverse: x pass (loader -> dst), then y and z (storer).
template <typename T, class Load, class Store>
cudaError_t inverse3(const Geom& g, const AxisTables<T>& tb, const int kinds[3], Load ld, T* dst, Store st,
                     cudaStream_t s) {
  cudaError_t e;
  if ((e = launch_pass<T, 0>(g, kinds[0], tb.t[0], ld, StoreField<T>{g, dst}, s)) != cudaSuccess) return e;
  return yz3(g, tb, kinds, dst, st, s);
}

// Inverse with a spectral multiplier: x pass on mul * src[i + di, j + dj,
// k + dk] -> dst through stx, then plain y and z passes in place (the z pass
// applies dk).
template <typename T, class Mul, class StX>
cudaError_t inverse3_mul(const Geom& g, const AxisTables<T>& tb, const int kinds[3], const T* src, Mul mul, int di,
                         int dj, int dk, StX stx, T* dst, cudaStream_t s) {
  cudaError_t e;
  if ((e = launch_mul_x_pass<T>(g, kinds[0], tb.t[0], src, mul, di, dj, stx, s)) != cudaSuccess) return e;
  return yz3(g, tb, kinds, dst, StoreField<T>{g, dst}, s, dk);
}

// Forward: z and y (loader -> dst), then x pass (storer).
template <typename T, class Load, class Store>
cudaError_t forward3(const Geom& g, const AxisTables<T>& tb, const int kinds[3], Load ld, T* dst, Store st,
                     cudaStream_t s) {
  cudaError_t e = cudaErrorNotSupported;
  if constexpr (std::is_same<Load, LoadField<T>>::value) e = launch_zpass<T>(g, kinds[2], tb.t[2], ld.src, dst, s);
  if (e == cudaErrorNotSupported) e = launch_pass<T, 2>(g, kinds[2], tb.t[2], ld, StoreField<T>{g, dst}, s);
  if (e != cudaSuccess) return e;
  if ((e = launch_pass<T, 1>(g, kinds[1], tb.t[1], LoadField<T>{g, dst}, StoreField<T>{g, dst}, s)) != cudaSuccess)
    return e;
  return launch_pass<T, 0>(g, kinds[0], tb.t[0], LoadField<T>{g, dst}, st, s);
}

// Two inverses of the same spectral source that differ only in their
// multiplier (same kinds and shifts): one dual x pass, then y and z of each.
template <typename T, class Mul, class Mul2>
cudaError_t inverse3_mul2(const Geom& g, const AxisTables<T>& tb, const int kinds[3], const T* src, Mul mul, Mul2 mul2,
                          int di, int dj, int dk, T* dst, T* dst2, cudaStream_t s) {
  cudaError_t e;
  if ((e = launch_mul_x_pass2<T>(g, kinds[0], tb.t[0], src, mul, mul2, di, dj, StoreField<T>{g, dst},
                                 StoreField<T>{g, dst2}, s)) != cudaSuccess)
    return e;
  if ((e = yz3(g, tb, kinds, dst, StoreField<T>{g, dst}, s, dk)) != cudaSuccess) return e;
  return yz3(g, tb, kinds, dst2, StoreField<T>{g, dst2}, s, dk);
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

#define QUASI_TRY(...)                        \
  do {                                        \
    cudaError_t e_ = (__VA_ARGS__);           \
    if (e_ != cudaSuccess) return e_;         \
  } while (0)

// Persistent elementwise grids: the blocks of `kern` resident per SM (from
// its occupancy at `threads` per block) times the SMs, so every block is
// running from the start and the grid-stride loops end together.
template <class K>
inline int ew_grid(K kern, int threads) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * tma_config().sms;
}
// Row-pack blocks: nz / V threads per row times the most rows that keep the
// block within 256 threads and a whole number of warps.
template <typename T>
inline dim3 row_block(int nz) {
  const int tx = nz / Pack<T>::V;
  int ty = tx >= 256 ? 1 : 256 / tx;
  while (ty > 1 && (tx * ty) % 32) --ty;
  return dim3(tx, ty);
}
#define QUASI_EW(kern, ...) kern<<<ew_grid(kern, 256), 256, 0, s>>>(__VA_ARGS__)
#define QUASI_EW_ON(kern, strm, ...) kern<<<ew_grid(kern, 256), 256, 0, strm>>>(__VA_ARGS__)

// z pass src -> dst: the TMA z kernel, else the general pass.  ks = 1
// transforms row[k + 1] (zero at the top), ks = 2 -mk[k] row[k + 1].
template <typename T>
cudaError_t zpass(const Geom& g, int kind, Tables<T> tb, T* src, T* dst, cudaStream_t s, int ks = 0,
                  const T* mk = nullptr) {
  const cudaError_t e = launch_zpass<T>(g, kind, tb, src, dst, s, ks, mk);
  if (e != cudaErrorNotSupported) return e;
  if (ks == 2)
    return launch_pass<T, 2, ShiftKMulLoad<T>, StoreField<T>>(g, kind, tb, ShiftKMulLoad<T>{g, src, mk},
                                                              StoreField<T>{g, dst}, s);
  return launch_pass<T, 2>(g, kind, tb, LoadField<T>{g, src}, StoreField<T>{g, dst}, s, ks);
}

// psi = iCT(psiq) (quasi.cpp:1963-1965) and grad psi (quasi.cpp:1120-1186) in
// double, in 9 axis passes instead of 12; with rho^ in place of psi^, rho =
// iCT(rho^) (quasi.cpp:1266-1268) and grad rho (quasi.cpp:1188-1232) the same way.  Each transform is separable and
// a multiplier or shift along one axis commutes with the passes along the
// others, so psi, grad_y and grad_z share the plain x pass X of psiq, and psi
// and grad_z share its plain y pass XY:
//   s:  X = x(psiq);  grad_y = z(y'(X));  XY = y(X);  psi = z(XY);
//       grad_z = z'(XY)
//   s2: grad_x = z(y(x'(psiq)))
// (a primed pass takes the shifted, scaled row and the odd kind: y' reads
// -vs_y[j] X[j + 1], z' -vs_z[k] XY[k + 1], x' -vs_x[i] psiq[i + 1]).  ev: a
// fork/join pair for the second stream (nullptr: everything on s).
template <typename T>
cudaError_t psi_and_grad(const StepCtx<T>& c, const AxisTables<double>& tb64, const double* psiq, double* psi,
                         double* gx, double* gy, double* gz, cudaStream_t s, cudaStream_t s2,
                         const cudaEvent_t* ev) {
  const Geom g = c.g;
  const bool two = s2 && ev;
  const cudaStream_t sb = two ? s2 : s;
  if (two) {
    QUASI_TRY(cudaEventRecord(ev[0], s));
    QUASI_TRY(cudaStreamWaitEvent(s2, ev[0], 0));
  }
  QUASI_TRY(inverse3_mul(g, tb64, kiSTx, psiq, MGrad<T, 0, false>{c}, 1, 0, 0, StoreField<double>{g, gx}, gx, sb));
  double* x = c.tmp64;
  QUASI_TRY(launch_pass<double, 0>(g, E01, tb64.t[0], LoadField<double>{g, psiq}, StoreField<double>{g, x}, s));
  QUASI_TRY(launch_mul_y_pass<double>(g, O01, tb64.t[1], x, MGrad<T, 1, false>{c}, StoreField<double>{g, gy}, s));
  QUASI_TRY(zpass<double>(g, E01, tb64.t[2], gy, gy, s));
  QUASI_TRY(launch_pass<double, 1>(g, E01, tb64.t[1], LoadField<double>{g, x}, StoreField<double>{g, x}, s));
  QUASI_TRY(zpass<double>(g, E01, tb64.t[2], x, psi, s));
  QUASI_TRY(zpass<double>(g, O01, tb64.t[2], x, gz, s, 2, c.vsz));
  if (two) {
    QUASI_TRY(cudaEventRecord(ev[1], s2));
    QUASI_TRY(cudaStreamWaitEvent(s, ev[1], 0));
  }
  return cudaSuccess;
}

// One time step, enqueued on `s` (captured into a CUDA graph by the caller).
// Independent transforms (the inverse transforms of psi^ and rho^, the three
// stress transforms, the five after the projection) are split over s and a
// second stream s2 between a fork and a join (ev[2i], ev[2i+1]; ev[6] orders
// the second stream's stress transform after the stress kernel, ev[7] the
// density chain after the gradients, ev[8], ev[9] the fork and join of psi
// and grad psi at the end, ev[10], ev[11] those of rho and grad rho in the
// FP64 form), so that in
// the captured graph one persistent pass kernel's last tiles overlap the next
// one's first loads.  s2 == nullptr: everything on s.
// tb64: the FP64 twiddles of the double transforms (the same tables as tb in
// the FP64 form).
template <typename T>
cudaError_t enqueue_step(const StepCtx<T>& c, const AxisTables<T>& tb, const AxisTables<double>& tb64, int* nloop_dev,
                         cudaStream_t s, cudaStream_t s2 = nullptr, const cudaEvent_t* ev = nullptr) {
  const Geom g = c.g;
  const size_t n = size_t(g.nx) * g.ny * g.nz;
  const cudaStream_t sb = s2 ? s2 : s;
  auto fork = [&](int i) -> cudaError_t {
    if (!s2) return cudaSuccess;
    cudaError_t e = cudaEventRecord(ev[2 * i], s);
    return e != cudaSuccess ? e : cudaStreamWaitEvent(s2, ev[2 * i], 0);
  };
  auto join = [&](int i) -> cudaError_t {
    if (!s2) return cudaSuccess;
    cudaError_t e = cudaEventRecord(ev[2 * i + 1], s2);
    return e != cudaSuccess ? e : cudaStreamWaitEvent(s, ev[2 * i + 1], 0);
  };
  bump_counter_kernel<<<1, 1, 0, s>>>(nloop_dev);
  QUASI_TRY(cudaGetLastError());
  auto st = [&](T* d) { return StoreField<T>{g, d}; };
  auto ld = [&](T* d) { return LoadField<T>{g, d}; };
  auto st64 = [&](double* d) { return StoreField<double>{g, d}; };
  if (c.variant == kQuasi) {
    // a4 gradients quasi.cpp:1120-1232: grad lap grad psi from the transform
    // copy of psi^, grad rho (grad psi in double is carried from the end of
    // the previous step, where it shares passes with psi)
    QUASI_TRY(fork(0));
    QUASI_TRY(inverse3_mul(g, tb, kiSTx, c.psiq_t, MGrad<T, 0, true>{c}, 1, 0, 0, st(c.ldx), c.ldx, s));
    QUASI_TRY(inverse3_mul(g, tb, kiSTy, c.psiq_t, MGrad<T, 1, true>{c}, 0, 1, 0, st(c.ldy), c.ldy, sb));
    QUASI_TRY(inverse3_mul(g, tb, kiSTz, c.psiq_t, MGrad<T, 2, true>{c}, 0, 0, 1, st(c.ldz), c.ldz, s));
    if constexpr (kStateCopy<T>) {   // (the FP64 form computed grad rho in the previous step)
      QUASI_TRY(inverse3_mul(g, tb, kiSTx, c.rhoq_t, MGrad<T, 0, false>{c}, 1, 0, 0, st(c.rdx), c.rdx, sb));
      QUASI_TRY(inverse3_mul(g, tb, kiSTy, c.rhoq_t, MGrad<T, 1, false>{c}, 0, 1, 0, st(c.rdy), c.rdy, s));
      QUASI_TRY(inverse3_mul(g, tb, kiSTz, c.rhoq_t, MGrad<T, 2, false>{c}, 0, 0, 1, st(c.rdz), c.rdz, sb));
    }
    // the density chain must not rewrite rho^ before the grad rho transforms
    // have read it: s waits for the second stream's share ...
    if (s2) {
      QUASI_TRY(cudaEventRecord(ev[7], s2));
      QUASI_TRY(cudaStreamWaitEvent(s, ev[7], 0));
    }
    // ... which then runs a3's prologue quasi.cpp:1036-1057 beside it
    QUASI_TRY(inverse3_mul2(g, tb, kiCT, c.psiq_t, MDf<T>{c}, MLap<T>{c}, 0, 0, 0, c.df, c.lap, sb));
    // a5 density + filter quasi.cpp:1237-1268 in double (rho doubles as the
    // scratch of its transform)
    QUASI_EW(rho_law_kernel<T>, c, n);
    QUASI_TRY(cudaGetLastError());
    const StRhoq sr{g, c.rhoq, c.scale, c.fx, c.fy, c.fz};
    if constexpr (kStateCopy<T>) {
      QUASI_TRY(forward3(g, tb64, kCT, LoadField<double>{g, c.rho}, c.rho, StRhoqCopy<T>{sr, c.rhoq_t}, s));
      QUASI_TRY(inverse3(g, tb64, kiCT, LoadField<double>{g, c.rhoq}, c.rho, st64(c.rho), s));
    } else {
      // rho and the next step's grad rho from the new rho^, sharing passes
      QUASI_TRY(forward3(g, tb64, kCT, LoadField<double>{g, c.rho}, c.rho, sr, s));
      QUASI_TRY(psi_and_grad(c, tb64, c.rhoq, c.rho, reinterpret_cast<double*>(c.rdnx),
                             reinterpret_cast<double*>(c.rdny), reinterpret_cast<double*>(c.rdnz), s, s2,
                             ev ? ev + 10 : nullptr));
    }
    QUASI_TRY(join(0));

  } else {
    // quasi-stb.cpp:1005-1038 (the unused dRho transform is elided; grad psi
    // is carried from the end of the previous step)
    QUASI_TRY(inverse3_mul(g, tb, kiCT, c.psiq_t, MSh<T>{c}, 0, 0, 0, st(c.sh), c.sh, s));
    // rho == 1, divv == 0, grad rho == 0 (rhoq never leaves 0): quasi-stb.cpp:1232
  }
  // a6 divv quasi.cpp:1273-1293 on the second stream, beside a7 the stress
  // quasi.cpp:1298-1330 (neither reads what the other writes; the projection
  // after the join reads both)
  QUASI_TRY(fork(1));
  if (c.variant == kQuasi) {
    QUASI_EW_ON(divv_kernel<T>, sb, c, n);
    QUASI_TRY(cudaGetLastError());
    QUASI_TRY(forward3(g, tb, kCT, ld(c.divv), c.divvq, st(c.divvq), sb));
  }
  QUASI_EW(stress_kernel<T>, c, n);
  QUASI_TRY(cudaGetLastError());
  if (s2) {   // Sy on the second stream once the stress is written
    QUASI_TRY(cudaEventRecord(ev[6], s));
    QUASI_TRY(cudaStreamWaitEvent(s2, ev[6], 0));
  }
  QUASI_TRY(forward3(g, tb, kSTy, ld(c.Sy), c.Sy, st(c.Sy), sb));
  QUASI_TRY(forward3(g, tb, kSTx, ld(c.Sx), c.Sx, st(c.Sx), s));
  QUASI_TRY(forward3(g, tb, kSTz, ld(c.Sz), c.Sz, st(c.Sz), s));
  QUASI_TRY(join(1));
  // a8 pressure, a9 velocity, a10 scaled divv quasi.cpp:1336-1900
  {
    const dim3 blk = row_block<T>(g.nz);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, project_kernel<T>, blk.x * blk.y, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    project_kernel<T><<<per_sm * tma_config().sms, blk, 0, s>>>(c);
  }
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(fork(2));
  if (c.variant == kQuasi) QUASI_TRY(inverse3(g, tb, kiCT, ld(c.p), c.p, st(c.p), s));
  QUASI_TRY(inverse3(g, tb, kiSTx, ld(c.vx), c.vx, st(c.vx), sb));
  QUASI_TRY(inverse3(g, tb, kiSTy, ld(c.vy), c.vy, st(c.vy), s));
  QUASI_TRY(inverse3(g, tb, kiSTz, ld(c.vz), c.vz, st(c.vz), sb));
  if (c.variant == kQuasi) QUASI_TRY(inverse3(g, tb, kiCT, ld(c.divv), c.divv, st(c.divv), s));
  QUASI_TRY(join(2));
  // a11 nonlinear term quasi.cpp:1905-1939
  QUASI_EW(nonlinear_kernel<T>, c, n);
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(forward3(g, tb, kCT, ld(c.Nq), c.Nq, st(c.Nq), s));
  // a12 update + iCT quasi.cpp:1944-1965
  {
    const dim3 blk = row_block<T>(g.nz);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, update_kernel<T>, blk.x * blk.y, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    update_kernel<T><<<per_sm * tma_config().sms, blk, 0, s>>>(c);
  }
  QUASI_TRY(cudaGetLastError());
  // psi = iCT(psiq_new) and grad psi in double for the next step (psi_old <-
  // psi by rotation)
  QUASI_TRY(psi_and_grad(c, tb64, c.psiq_new, c.psi_new, c.gx, c.gy, c.gz, s, s2, ev ? ev + 8 : nullptr));
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
    c.rhoq[id] = 0.0;
    if constexpr (kStateCopy<T>) {
      c.rhoq_t[id] = T(0);
    } else {   // grad rho of rho^ = 0, both rotation buffers
      c.rdx[id] = c.rdy[id] = c.rdz[id] = T(0);
      c.rdnx[id] = c.rdny[id] = c.rdnz[id] = T(0);
    }
    c.rho_old[id] = 0.0;
    c.vx[id] = T(0);
    c.vy[id] = T(0);
    c.vz[id] = T(0);
    c.p[id] = T(0);
    c.rho[id] = c.variant == kQuasi ? 0.0 : 1.0;
  }
}

// double field -> storage type (the FP32 form's copy of psi^ after the pre-loop)
template <typename T>
__global__ void to_storage_kernel(const double* src, T* dst, size_t n) {
  for (size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x; id < n; id += size_t(gridDim.x) * blockDim.x)
    dst[id] = T(src[id]);
}

// The projection psiq = scale CT(psi), psi = iCT(psiq) runs in double in both
// forms (quasi_set_psi leaves the initial psi in c.psi).
template <typename T>
cudaError_t enqueue_init(const StepCtx<T>& c, const AxisTables<T>& tb, const AxisTables<double>& tb64, int* nloop_dev,
                         cudaStream_t s) {
  const Geom g = c.g;
  const size_t n = size_t(g.nx) * g.ny * g.nz;
  QUASI_TRY(forward3(g, tb64, kCT, LoadField<double>{g, c.psi}, c.psiq, ScaleStore<double>{g, c.psiq, c.scale}, s));
  if constexpr (kStateCopy<T>) {
    to_storage_kernel<T><<<592, 256, 0, s>>>(c.psiq, c.psiq_t, n);
    QUASI_TRY(cudaGetLastError());
  }
  QUASI_TRY(psi_and_grad(c, tb64, c.psiq, c.psi, c.gx, c.gy, c.gz, s, nullptr, nullptr));
  QUASI_TRY(forward3(g, tb, kCT, LdInitN<T>{c}, c.Nq_old, StoreField<T>{g, c.Nq_old}, s));
  init_state_kernel<T><<<592, 256, 0, s>>>(c, n);
  QUASI_TRY(cudaGetLastError());
  QUASI_TRY(cudaMemsetAsync(nloop_dev, 0, sizeof(int), s));
  return cudaSuccess;
}

}  // namespace quasi
