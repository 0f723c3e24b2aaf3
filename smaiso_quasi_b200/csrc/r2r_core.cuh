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

QHD constexpr RadixPlan radix_plan(int n) {
  RadixPlan p{0, {0, 0, 0, 0, 0, 0}};
  int m = n;
  // prefer 16 and 8 (fewer stages), keep the 3s last
  while (m % 16 == 0 && m != 32 && p.n_stages < 6) { p.r[p.n_stages++] = 16; m /= 16; }
  while (m % 8 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 8; m /= 8; }
  while (m % 4 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 4; m /= 4; }
  while (m % 2 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 2; m /= 2; }
  while (m % 3 == 0 && p.n_stages < 6) { p.r[p.n_stages++] = 3; m /= 3; }
  if (m != 1) p.n_stages = -1;
  return p;
}

QHD constexpr bool size_supported(int n) { return n >= 4 && (n % 2) == 0 && radix_plan(n).n_stages > 0; }

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
// In-place tile transform.
//
// Tile: P = 2G real pencils of length N at buf[r * LD + n] (reals), LD = N + 1.
// Complex pencil g (LD complex elements) occupies exactly the bytes of real
// pencils 2g and 2g+1, so the whole transform runs in ONE buffer: every stage
// reads all its inputs into registers, the CTA synchronises, then writes.
// Work items are mapped pencil-fastest (g = w % G) so that neighbouring
// threads touch the same offset of neighbouring pencils; the odd stride LD
// keeps those in distinct shared-memory banks.
//
// The Makhoul reordering is folded into the first stage's reads (forward
// kinds, and the inverse kinds' V_k = e^{i pi k/2N}(y_k - i y_{N-k})) and the
// inverse un-reordering into the last stage's writes; the forward kinds'
// pairing of Z_k with Z_{N-k} is one extra read/write phase.
// ---------------------------------------------------------------------------
QHD constexpr int tile_ld(int n) { return n + 1; }

template <typename T, int N, int G, int NT>
struct TileFFT {
  static constexpr RadixPlan plan = radix_plan(N);
  static constexpr int LD = tile_ld(N);
  static_assert(plan.n_stages > 0, "unsupported transform length");

  // butterflies a thread owns in a radix-R stage
  template <int R> static constexpr int per_thread() { return (G * (N / R) + NT - 1) / NT; }
  static constexpr int kMaxRegs = 16;   // complex values a thread holds in any phase

  // ---- stage input element e of complex pencil g --------------------------
  // first stage: the packed complex sequence is formed from the real tile
  QHD static Cx<T> first_input(const T* buf, int kind, int g, int e, Tables<T> tb) {
    const T* a = buf + (2 * g) * LD;
    const T* b = a + LD;
    if (is_forward(kind)) {
      // v_e = x_{2e} (e < N/2), x_{2(N-1-e)+1} (e >= N/2); DST-II negates odd x
      int src;
      T sgn = T(1);
      if (e < N / 2) src = 2 * e;
      else { src = 2 * (N - 1 - e) + 1; if (kind == O10) sgn = T(-1); }
      return Cx<T>{sgn * a[src], sgn * b[src]};
    }
    // inverse: conj( e^{+i pi k/2N} [(ya_k - i ya_{N-k}) + i (yb_k - i yb_{N-k})] ), y_N = 0,
    // input reversed for DST-III
    const int k = e;
    const bool rev = kind == O01;
    const int ik = rev ? N - 1 - k : k;
    const T ak = a[ik], bk = b[ik];
    T an = T(0), bn = T(0);
    if (k) {
      const int in_ = rev ? k - 1 : N - k;   // index of y_{N-k} (reversed: N-1-(N-k))
      an = a[in_];
      bn = b[in_];
    }
    const Cx<T> q = tb.quarter[k];
    const Cx<T> ec = {q.x, -q.y};
    const Cx<T> va = cmul(ec, Cx<T>{ak, -an});
    const Cx<T> vb = cmul(ec, Cx<T>{bk, -bn});
    return Cx<T>{va.x - vb.y, -(va.y + vb.x)};
  }

  // last stage of an inverse kind: FFT output F_k -> u_k = conj(F_k) -> the
  // two real pencils at the un-reordered positions (DST-III negates odd x)
  QHD static void last_output_inverse(T* buf, int kind, int g, int k, Cx<T> f) {
    T* a = buf + (2 * g) * LD;
    T* b = a + LD;
    int dst;
    T sgn = T(1);
    if (k < N / 2) dst = 2 * k;
    else { dst = 2 * (N - 1 - k) + 1; if (kind == O01) sgn = T(-1); }
    a[dst] = sgn * f.x;
    b[dst] = -sgn * f.y;
  }

  // ---- one Stockham stage, split into its read and write halves -----------
  template <int R>
  struct StageRegs {
    Cx<T> v[per_thread<R>()][R];
  };

  template <int R>
  QHD static void stage_read(int tid, const T* buf, int kind, int n, int s, bool first, Tables<T> tb,
                             StageRegs<R>& r) {
    const Cx<T>* cb = reinterpret_cast<const Cx<T>*>(buf);
    const int m = n / R;
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * (N / R)) break;
      const int g = w % G, bfl = w / G;
      const int p = bfl / s, q = bfl - p * s;
#pragma unroll
      for (int t = 0; t < R; ++t) {
        const int e = q + s * (p + t * m);
        r.v[c][t] = first ? first_input(buf, kind, g, e, tb) : cb[g * LD + e];
      }
      Dft<T, R>::run(r.v[c]);
      const int step = (N / n) * p;   // W_n^{p u} = root[(N/n) p u], (N/n) p u < N
#pragma unroll
      for (int u = 1; u < R; ++u)
        if (p) r.v[c][u] = cmul(r.v[c][u], tb.root[step * u]);
    }
  }

  template <int R>
  QHD static void stage_write(int tid, T* buf, int kind, int n, int s, bool last, const StageRegs<R>& r) {
    Cx<T>* cb = reinterpret_cast<Cx<T>*>(buf);
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * (N / R)) break;
      const int g = w % G, bfl = w / G;
      const int p = bfl / s, q = bfl - p * s;
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int k = q + s * (R * p + u);
        if (last && !is_forward(kind)) last_output_inverse(buf, kind, g, k, r.v[c][u]);
        else cb[g * LD + k] = r.v[c][u];
      }
    }
  }

  // ---- forward kinds: pair Z_k with Z_{N-k} ---------------------------------
  static constexpr int kPairs = N / 2 + 1;   // k = 0 .. N/2
  static constexpr int kUnpackPerThread = (G * kPairs + NT - 1) / NT;
  struct UnpackRegs {
    T ya[kUnpackPerThread][2], yb[kUnpackPerThread][2];
  };

  QHD static void unpack_read(int tid, const T* buf, int kind, Tables<T> tb, UnpackRegs& r) {
    const Cx<T>* cb = reinterpret_cast<const Cx<T>*>(buf);
    (void)kind;
#pragma unroll
    for (int c = 0; c < kUnpackPerThread; ++c) {
      const int w = tid + c * NT;
      if (w >= G * kPairs) break;
      const int g = w % G, k = w / G;
      const int kn = (N - k) % N;
      const Cx<T> z0 = cb[g * LD + k], z1 = cb[g * LD + kn];
      // y(k) from (Z_k, Z_{N-k}); y(N-k) from (Z_{N-k}, Z_k)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const Cx<T> zk = h ? z1 : z0;
        const Cx<T> zr = conj(h ? z0 : z1);
        const int kk = h ? kn : k;
        const Cx<T> va = zk + zr;
        const Cx<T> d = zk - zr;
        const Cx<T> vb = {d.y, -d.x};
        const Cx<T> qk = tb.quarter[kk];
        r.ya[c][h] = qk.x * va.x - qk.y * va.y;
        r.yb[c][h] = qk.x * vb.x - qk.y * vb.y;
      }
    }
  }

  QHD static void unpack_write(int tid, T* buf, int kind, const UnpackRegs& r) {
#pragma unroll
    for (int c = 0; c < kUnpackPerThread; ++c) {
      const int w = tid + c * NT;
      if (w >= G * kPairs) break;
      const int g = w % G, k = w / G;
      T* a = buf + (2 * g) * LD;
      T* b = a + LD;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (h && (k == 0 || k == N / 2)) continue;   // self-paired
        const int kk = h ? N - k : k;
        const int dst = kind == O10 ? N - 1 - kk : kk;
        a[dst] = r.ya[c][h];
        b[dst] = r.yb[c][h];
      }
    }
  }
};

// Runs the whole in-place transform of the tile in `buf`.  `ex.phase2(rd, wr,
// tid, regs)` runs rd(tid, regs), synchronises the CTA, runs wr(tid, regs) and
// synchronises again on the device; the CPU test runs rd for every thread
// (each with its own registers) before any wr.
template <typename T, int N, int G, int NT, int ST, class Exec>
QHD void r2r_stages(Exec& ex, int tid, int kind, T* buf, Tables<T> tb, int n, int s) {
  using F = TileFFT<T, N, G, NT>;
  if constexpr (ST < F::plan.n_stages) {
    constexpr int R = F::plan.r[ST];
    constexpr bool first = ST == 0, last = ST == F::plan.n_stages - 1;
    using Regs = typename F::template StageRegs<R>;
    Regs regs;
    ex.phase2([&](int t, Regs& rg) { F::template stage_read<R>(t, buf, kind, n, s, first, tb, rg); },
              [&](int t, Regs& rg) { F::template stage_write<R>(t, buf, kind, n, s, last, rg); }, tid, regs);
    r2r_stages<T, N, G, NT, ST + 1>(ex, tid, kind, buf, tb, n / R, s * R);
  }
}

template <typename T, int N, int G, int NT, class Exec>
QHD void r2r_tile_inplace(Exec& ex, int tid, int kind, T* buf, Tables<T> tb) {
  using F = TileFFT<T, N, G, NT>;
  r2r_stages<T, N, G, NT, 0>(ex, tid, kind, buf, tb, N, 1);
  if (is_forward(kind)) {
    typename F::UnpackRegs regs;
    ex.phase2([&](int t, typename F::UnpackRegs& rg) { F::unpack_read(t, buf, kind, tb, rg); },
              [&](int t, typename F::UnpackRegs& rg) { F::unpack_write(t, buf, kind, rg); }, tid, regs);
  }
}

}  // namespace quasi
