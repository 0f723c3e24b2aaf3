// Batched 1-D real-to-real transforms of FFTW's kinds on pencils staged in
// shared memory: the building block of every 3-D transform of the step.
//
// Kinds (FFTW 3.3 unnormalised definitions, the ones quasi.cpp:449-495 plans):
//   E10 REDFT10  y_k = 2 sum_n x_n cos(pi k (2n+1) / 2N)             (DCT-II)
//   E01 REDFT01  y_k = x_0 + 2 sum_{n>=1} x_n cos(pi n (2k+1) / 2N)  (DCT-III)
//   O10 RODFT10  y_k = 2 sum_n x_n sin(pi (k+1)(2n+1) / 2N)          (DST-II)
//   O01 RODFT01  y_k = (-1)^k x_{N-1} + 2 sum_{n<N-1} x_n sin(pi (n+1)(2k+1)/2N)
// Algorithm: Makhoul's reordering turns each kind into one complex DFT of
// length N; two real pencils share one complex DFT (real and imaginary part).
//   O10(x)_k = E10((-1)^n x_n)_{N-1-k},   O01(y)_k = (-1)^k E01(reverse y)_k.
// The complex DFT is a mixed-radix (16, 8, 4, 3, 2) Stockham FFT, one
// butterfly per thread per stage, ping-ponging between two shared buffers.
//
// Every phase is a __host__ __device__ function over a flat work index, so the
// exact device indexing also runs (serially) in the CPU unit test.
#pragma once
#include <cstdint>
#include <type_traits>

#ifdef __CUDACC__
#define QHD __host__ __device__ __forceinline__
#else
#define QHD inline
#endif

namespace quasi {

template <typename T>
struct Cx {
  T x, y;
};

template <typename T> QHD Cx<T> cx(T a, T b) { return Cx<T>{a, b}; }
template <typename T> QHD Cx<T> operator+(Cx<T> a, Cx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> QHD Cx<T> operator-(Cx<T> a, Cx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T> QHD Cx<T> cmul(Cx<T> a, Cx<T> b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <typename T> QHD Cx<T> cscale(Cx<T> a, T s) { return {a.x * s, a.y * s}; }
template <typename T> QHD Cx<T> conj(Cx<T> a) { return {a.x, -a.y}; }
template <typename T> QHD Cx<T> mul_mi(Cx<T> a) { return {a.y, -a.x}; }   // -i * a

// FP32 complex adds and scales on sm_100's packed FP32x2 instructions (one
// FADD2 / FMUL2 per complex add or scale; each lane rounds as the scalar
// instruction does, so results are unchanged).  Complex products stay scalar:
// packing their operands ((a.x, a.x), (b.y, b.x), ...) costs register moves
// that outweigh the saving.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
__device__ __forceinline__ float2 f2(Cx<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ Cx<float> cf(float2 a) { return Cx<float>{a.x, a.y}; }
__device__ __forceinline__ Cx<float> operator+(Cx<float> a, Cx<float> b) { return cf(__fadd2_rn(f2(a), f2(b))); }
__device__ __forceinline__ Cx<float> operator-(Cx<float> a, Cx<float> b) {
  return cf(__fadd2_rn(f2(a), make_float2(-b.x, -b.y)));
}
__device__ __forceinline__ Cx<float> cscale(Cx<float> a, float s) { return cf(__fmul2_rn(f2(a), make_float2(s, s))); }
#endif

enum Kind : int { E10 = 0, E01 = 1, O10 = 2, O01 = 3 };
QHD bool is_forward(int kind) { return kind == E10 || kind == O10; }
QHD bool is_sine(int kind) { return kind == O10 || kind == O01; }

// ---------------------------------------------------------------------------
// Radix plans: N = 2^a 3^b, 8 <= N <= 1024, stages in order of use.
// ---------------------------------------------------------------------------
struct RadixPlan {
  int n_stages;
  int r[6];
};

QHD constexpr RadixPlan radix_plan(int n, int max_radix = 16) {
  RadixPlan p{0, {0, 0, 0, 0, 0, 0}};
  int m = n;
  // prefer the largest radix allowed (fewer stages), keep the 3s last
  while (max_radix >= 16 && m % 16 == 0 && m != 32 && p.n_stages < 6) { p.r[p.n_stages++] = 16; m /= 16; }
  while (m % 8 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 8; m /= 8; }
  while (m % 4 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 4; m /= 4; }
  while (m % 2 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 2; m /= 2; }
  while (m % 3 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 3; m /= 3; }
  if (m != 1) p.n_stages = -1;
  return p;
}

QHD constexpr bool size_supported(int n) { return n >= 4 && (n % 2) == 0 && radix_plan(n).n_stages > 0; }

// Stride s (product of the radices before stage st) and sub-length n = N / s.
QHD constexpr int stage_stride(int n, int st, int max_radix) {
  int s = 1;
  for (int i = 0; i < st; ++i) s *= radix_plan(n, max_radix).r[i];
  return s;
}

// Largest radix per element type: a radix-16 butterfly holds 16 complex values
// in registers (64 registers in double), so double stops at 8.
template <typename T> QHD constexpr int max_radix() { return sizeof(T) == 8 ? 8 : 16; }

// ---------------------------------------------------------------------------
// Small forward DFT codelets, exp(-2 pi i tu / R)
// ---------------------------------------------------------------------------
template <typename T, int R> struct Dft;

template <typename T> struct Dft<T, 2> {
  QHD static void run(Cx<T>* a) {
    Cx<T> t = a[0];
    a[0] = t + a[1];
    a[1] = t - a[1];
  }
};

template <typename T> struct Dft<T, 3> {
  QHD static void run(Cx<T>* a) {
    const T c = T(-0.5), s = T(0.86602540378443864676372317075294);
    Cx<T> t1 = a[1] + a[2], t2 = a[1] - a[2];
    Cx<T> base = a[0] + cscale(t1, c);
    Cx<T> rot = {s * t2.y, -s * t2.x};
    a[0] = a[0] + t1;
    a[1] = base + rot;
    a[2] = base - rot;
  }
};

template <typename T> struct Dft<T, 4> {
  QHD static void run(Cx<T>* a) {
    Cx<T> t0 = a[0] + a[2], t1 = a[0] - a[2], t2 = a[1] + a[3], t3 = mul_mi(a[1] - a[3]);
    a[0] = t0 + t2;
    a[2] = t0 - t2;
    a[1] = t1 + t3;
    a[3] = t1 - t3;
  }
};

// W_16^m for m = 0..9 (cos, -sin): the twiddles of the 4x4 and 2x4 splits
template <typename T> QHD Cx<T> w16(int m) {
  const T c1 = T(0.92387953251128675612818318939679), s1 = T(0.38268343236508977172845998403040);
  const T h = T(0.70710678118654752440084436210485);
  switch (m) {
    case 0: return {T(1), T(0)};
    case 1: return {c1, -s1};
    case 2: return {h, -h};
    case 3: return {s1, -c1};
    case 4: return {T(0), T(-1)};
    case 5: return {-s1, -c1};
    case 6: return {-h, -h};
    case 7: return {-c1, -s1};
    case 8: return {T(-1), T(0)};
    default: return {-c1, s1};   // m = 9
  }
}

// R = R1 * R2 split: X[k1 + R1 k2] = sum_n2 W_R2^{n2 k2} W_R^{n2 k1} sum_n1 a[R2 n1 + n2] W_R1^{n1 k1}
template <typename T, int R1, int R2> struct DftSplit {
  QHD static void run(Cx<T>* a) {
    Cx<T> t[R2][R1];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) t[n2][n1] = a[R2 * n1 + n2];
      Dft<T, R1>::run(t[n2]);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        const int m = n2 * k1 * (16 / (R1 * R2));
        if (m) t[n2][k1] = cmul(t[n2][k1], w16<T>(m));
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      Cx<T> u[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) u[n2] = t[n2][k1];
      Dft<T, R2>::run(u);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) a[k1 + R1 * k2] = u[k2];
    }
  }
};

template <typename T> struct Dft<T, 8> {
  QHD static void run(Cx<T>* a) { DftSplit<T, 2, 4>::run(a); }
};
template <typename T> struct Dft<T, 16> {
  QHD static void run(Cx<T>* a) { DftSplit<T, 4, 4>::run(a); }
};

// ---------------------------------------------------------------------------
// Tables (device or host memory), computed on the host in long double:
//   root[t]    = exp(-2 pi i t / N),       t < N
//   quarter[k] = exp(-i pi k / (2N)),      k < N
// ---------------------------------------------------------------------------
template <typename T>
struct Tables {
  const Cx<T>* root;
  const Cx<T>* quarter;
};

// ---------------------------------------------------------------------------
// Tile transform with pluggable input and output.
//
// G complex pencils of length N live in a shared buffer `cb` (pencil g at
// cb[g * LD + e], LD = N + 1) between stages.  Complex pencil g carries the
// real pencils 2g (real part) and 2g+1 (imaginary part).
//   Src::pair(g, n, a, b)  the two reals of pencils 2g, 2g+1 at position n
//   Snk::put(g, n, a, b)   store the two reals of pencils 2g, 2g+1 at n
// The first stage reads through Src with the Makhoul reordering folded in;
// the last stage of an inverse kind writes through Snk with the
// un-reordering folded in; a forward kind pairs Z_k with Z_{N-k} from the
// shared buffer and writes through Snk.  When Src/Snk are the shared buffer
// itself (in-place, real pencil r at r * LD) every read half is separated
// from its write half by a barrier; when they are global memory the first
// stage needs no barrier before its shared writes and an inverse kind's last
// stage none before its global stores.
//
// Work items are mapped pencil-fastest (g = w % G) so that neighbouring
// threads touch the same offset of neighbouring pencils: conflict-free with
// the odd stride LD in shared memory and coalesced (adjacent k) in global.
// ---------------------------------------------------------------------------
QHD constexpr int tile_ld(int n) { return n + 1; }

template <typename T>
struct SmemSrc {
  const T* buf;
  int ld;
  QHD void pair(int g, int n, T& a, T& b) const {
    a = buf[(2 * g) * ld + n];
    b = buf[(2 * g + 1) * ld + n];
  }
};

template <typename T>
struct SmemSnk {
  T* buf;
  int ld;
  QHD void put(int g, int n, T a, T b) const {
    buf[(2 * g) * ld + n] = a;
    buf[(2 * g + 1) * ld + n] = b;
  }
};

// Tile layout between stages: complex element e of pencil g at
// cb[g * GS + e * ES], pencil-major with the odd stride LD = N + 1.
template <int N>
struct PencilMajor {
  static constexpr int GS = tile_ld(N), ES = 1;
};

template <typename T, int N, int G, int NT, class L = PencilMajor<N>>
struct TileFFT {
  static constexpr RadixPlan plan = radix_plan(N, max_radix<T>());
  static constexpr int LD = tile_ld(N);
  static_assert(plan.n_stages > 0, "unsupported transform length");
  QHD static constexpr int at(int g, int e) { return g * L::GS + e * L::ES; }

  // butterflies a thread owns in a radix-R stage
  template <int R> static constexpr int per_thread() { return (G * (N / R) + NT - 1) / NT; }

  // first stage: the packed complex input e of pencil g, formed from Src
  template <class Src>
  QHD static Cx<T> first_input(const Src& src, int kind, int g, int e, Tables<T> tb) {
    if (is_forward(kind)) {
      // v_e = x_{2e} (e < N/2), x_{2(N-1-e)+1} (e >= N/2); DST-II negates odd x
      int n;
      T sgn = T(1);
      if (e < N / 2) n = 2 * e;
      else { n = 2 * (N - 1 - e) + 1; if (kind == O10) sgn = T(-1); }
      T a, b;
      src.pair(g, n, a, b);
      return Cx<T>{sgn * a, sgn * b};
    }
    // inverse: conj( e^{+i pi k/2N} [(ya_k - i ya_{N-k}) + i (yb_k - i yb_{N-k})] ), y_N = 0,
    // input reversed for DST-III
    const int k = e;
    const bool rev = kind == O01;
    T ak, bk, an = T(0), bn = T(0);
    src.pair(g, rev ? N - 1 - k : k, ak, bk);
    if (k) src.pair(g, rev ? k - 1 : N - k, an, bn);
    const Cx<T> q = tb.quarter[k];
    const Cx<T> ec = {q.x, -q.y};
    const Cx<T> va = cmul(ec, Cx<T>{ak, -an});
    const Cx<T> vb = cmul(ec, Cx<T>{bk, -bn});
    return Cx<T>{va.x - vb.y, -(va.y + vb.x)};
  }

  template <int R>
  struct StageRegs {
    Cx<T> v[per_thread<R>()][R];
  };

  template <int R, int n, int s, class Src>
  QHD static void stage_read(int tid, const Cx<T>* cb, const Src& src, int kind, bool first, Tables<T> tb,
                             StageRegs<R>& r) {
    constexpr int m = n / R;
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * (N / R)) break;
      const int g = w % G, bfl = w / G;
      const int p = bfl / s, q = bfl - p * s;
#pragma unroll
      for (int t = 0; t < R; ++t) {
        const int e = q + s * (p + t * m);
        r.v[c][t] = first ? first_input(src, kind, g, e, tb) : cb[at(g, e)];
      }
      Dft<T, R>::run(r.v[c]);
      const int step = (N / n) * p;   // W_n^{p u} = root[(N/n) p u], (N/n) p u < N
#pragma unroll
      for (int u = 1; u < R; ++u)
        if (p) r.v[c][u] = cmul(r.v[c][u], tb.root[step * u]);
    }
  }

  template <int R, int s, class Snk>
  QHD static void stage_write(int tid, Cx<T>* cb, const Snk& snk, int kind, bool last, const StageRegs<R>& r) {
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * (N / R)) break;
      const int g = w % G, bfl = w / G;
      const int p = bfl / s, q = bfl - p * s;
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int k = q + s * (R * p + u);
        const Cx<T> f = r.v[c][u];
        if (last && !is_forward(kind)) {
          // u_k = conj(F_k) -> x_{2k} (k < N/2) or x_{2(N-1-k)+1}; DST-III negates odd x
          int n;
          T sgn = T(1);
          if (k < N / 2) n = 2 * k;
          else { n = 2 * (N - 1 - k) + 1; if (kind == O01) sgn = T(-1); }
          snk.put(g, n, sgn * f.x, -sgn * f.y);
        } else {
          cb[at(g, k)] = f;
        }
      }
    }
  }

  // forward kinds: y(k) and y(N-k) from the pair (Z_k, Z_{N-k}), k = 0..N/2
  static constexpr int kPairs = N / 2 + 1;
  static constexpr int kUnpackPerThread = (G * kPairs + NT - 1) / NT;
  struct UnpackRegs {
    T ya[kUnpackPerThread][2], yb[kUnpackPerThread][2];
  };

  QHD static void unpack_read(int tid, const Cx<T>* cb, Tables<T> tb, UnpackRegs& r) {
#pragma unroll
    for (int c = 0; c < kUnpackPerThread; ++c) {
      const int w = tid + c * NT;
      if (w >= G * kPairs) break;
      const int g = w % G, k = w / G;
      const int kn = (N - k) % N;
      const Cx<T> z0 = cb[at(g, k)], z1 = cb[at(g, kn)];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const Cx<T> zk = h ? z1 : z0;
        const Cx<T> zr = conj(h ? z0 : z1);
        const int kk = h ? kn : k;
        const Cx<T> va = zk + zr;            // 2 V_a
        const Cx<T> d = zk - zr;
        const Cx<T> vb = {d.y, -d.x};        // 2 V_b
        const Cx<T> qk = tb.quarter[kk];     // y = 2 Re(quarter_k V)
        r.ya[c][h] = qk.x * va.x - qk.y * va.y;
        r.yb[c][h] = qk.x * vb.x - qk.y * vb.y;
      }
    }
  }

  template <class Snk>
  QHD static void unpack_write(int tid, const Snk& snk, int kind, const UnpackRegs& r) {
#pragma unroll
    for (int c = 0; c < kUnpackPerThread; ++c) {
      const int w = tid + c * NT;
      if (w >= G * kPairs) break;
      const int g = w % G, k = w / G;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (h && (k == 0 || k == N / 2)) continue;   // self-paired
        const int kk = h ? N - k : k;
        snk.put(g, kind == O10 ? N - 1 - kk : kk, r.ya[c][h], r.yb[c][h]);
      }
    }
  }
};

// Stage recursion.  `ex.phase(rd, wr, tid, regs, mid, after)` runs rd(tid,
// regs), a barrier when `mid`, wr(tid, regs), a barrier when `after`; the CPU
// test runs rd for every thread before any wr.
struct NoHook {
  QHD void operator()() const {}
};

// A source whose bytes ARE the tile (`kAliasesTile`): the first stage then
// reads everything before it writes, like an in-place stage.
template <class S, class = void> struct SrcAliasesTile {
  static constexpr bool value = false;
};
template <class S> struct SrcAliasesTile<S, std::void_t<decltype(S::kAliasesTile)>> {
  static constexpr bool value = S::kAliasesTile;
};
// The same for a sink: the last stage (or the unpack) then reads everything
// before it writes.
template <class S> using SnkAliasesTile = SrcAliasesTile<S>;

// `hook()` runs on every thread right after the first stage's closing barrier
// (the moment the first stage's input is no longer needed).
template <typename T, int N, int G, int NT, int ST, bool INPLACE, class L, class Exec, class Src, class Snk,
          class Hook>
QHD void r2r_stages(Exec& ex, int tid, int kind, Cx<T>* cb, const Src& src, const Snk& snk, Tables<T> tb,
                    const Hook& hook) {
  using F = TileFFT<T, N, G, NT, L>;
  if constexpr (ST < F::plan.n_stages) {
    constexpr int R = F::plan.r[ST];
    constexpr int s = stage_stride(N, ST, max_radix<T>()), n = N / s;
    constexpr bool first = ST == 0, last = ST == F::plan.n_stages - 1;
    using Regs = typename F::template StageRegs<R>;
    Regs regs;
    // a read half must finish before its write half only if the writes can
    // land on data other threads still read: always when Src/Snk are the
    // shared buffer; otherwise only for middle stages and a forward kind's
    // last stage (both write the shared buffer they read)
    const bool global_out = last && !is_forward(kind);
    const bool mid = INPLACE || (first ? SrcAliasesTile<Src>::value : (!global_out || SnkAliasesTile<Snk>::value));
    // a write half must be visible before the next read half; an inverse
    // kind's last stage writing to global memory is followed by nothing
    const bool after = !last || is_forward(kind) || INPLACE;
    ex.phase([&](int t, Regs& rg) { F::template stage_read<R, n, s>(t, cb, src, kind, first, tb, rg); },
             [&](int t, Regs& rg) { F::template stage_write<R, s>(t, cb, snk, kind, last, rg); }, tid, regs, mid,
             after);
    if constexpr (first) {
      if (!after) ex.sync();   // the hook may recycle the first stage's input
      hook();
    }
    r2r_stages<T, N, G, NT, ST + 1, INPLACE, L>(ex, tid, kind, cb, src, snk, tb, hook);
  }
}

template <typename T, int N, int G, int NT, bool INPLACE, class L = PencilMajor<N>, class Exec, class Src, class Snk,
          class Hook = NoHook>
QHD void r2r_tile(Exec& ex, int tid, int kind, Cx<T>* cb, const Src& src, const Snk& snk, Tables<T> tb,
                  const Hook& hook = Hook()) {
  using F = TileFFT<T, N, G, NT, L>;
  r2r_stages<T, N, G, NT, 0, INPLACE, L>(ex, tid, kind, cb, src, snk, tb, hook);
  if (is_forward(kind)) {
    typename F::UnpackRegs regs;
    ex.phase([&](int t, typename F::UnpackRegs& rg) { F::unpack_read(t, cb, tb, rg); },
             [&](int t, typename F::UnpackRegs& rg) { F::unpack_write(t, snk, kind, rg); }, tid, regs,
             INPLACE || SnkAliasesTile<Snk>::value, INPLACE);
  }
}

// In-place transform of P = 2G real pencils held in `buf` (real pencil r at
// buf[r * LD + n]); the complex pencils overlay the same bytes.
template <typename T, int N, int G, int NT, class Exec>
QHD void r2r_tile_inplace(Exec& ex, int tid, int kind, T* buf, Tables<T> tb) {
  constexpr int LD = tile_ld(N);
  r2r_tile<T, N, G, NT, true>(ex, tid, kind, reinterpret_cast<Cx<T>*>(buf), SmemSrc<T>{buf, LD}, SmemSnk<T>{buf, LD},
                              tb);
}

}  // namespace quasi
