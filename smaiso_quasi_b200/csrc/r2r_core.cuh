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

// One Stockham stage: src -> dst, n = current sub-length, s = stride, radix R.
// Work items: G complex pencils x (N / R) butterflies, pencil index fastest so
// that neighbouring threads touch the same offset of neighbouring pencils
// (pencil stride ld = N + 1 keeps those in distinct shared-memory banks).
template <typename T, int N, int R>
QHD void stockham_stage(int w, int G, const Cx<T>* src, Cx<T>* dst, int n, int s, int ld, Tables<T> tb) {
  const int g = w % G, b = w / G;
  const int m = n / R;
  const int p = b / s, q = b - p * s;
  const Cx<T>* sp = src + g * ld;
  Cx<T>* dp = dst + g * ld;
  Cx<T> a[R];
#pragma unroll
  for (int t = 0; t < R; ++t) a[t] = sp[q + s * (p + t * m)];
  Dft<T, R>::run(a);
  const int step = (N / n) * p;   // W_n^{p u} = root[(N/n) p u]
#pragma unroll
  for (int u = 0; u < R; ++u) {
    Cx<T> v = a[u];
    if (u && p) v = cmul(v, tb.root[step * u]);   // step*u <= (m-1)(R-1)N/n < N
    dp[q + s * (R * p + u)] = v;
  }
}

// ---------------------------------------------------------------------------
// The tile: P real pencils of length N at rt[p * ldr + n] (real layout) and
// G = P/2 complex pencils at cb[g * ldc + n].  Both buffers are the same
// byte size and alternate roles.
// ---------------------------------------------------------------------------

// (1) forward kinds: real tile -> packed complex (Makhoul reorder, DST sign)
template <typename T, int N>
QHD void fwd_pack(int w, int G, int kind, const T* rt, int ldr, Cx<T>* cb, int ldc) {
  // w in [0, G * N/2)
  const int g = w % G, t = w / G;
  const T* a = rt + (2 * g) * ldr;
  const T* b = rt + (2 * g + 1) * ldr;
  T a0 = a[2 * t], a1 = a[2 * t + 1], b0 = b[2 * t], b1 = b[2 * t + 1];
  if (kind == O10) { a1 = -a1; b1 = -b1; }
  cb[g * ldc + t] = Cx<T>{a0, b0};
  cb[g * ldc + N - 1 - t] = Cx<T>{a1, b1};
}

// (2) forward kinds: complex spectrum -> two real pencils
template <typename T, int N>
QHD void fwd_unpack(int w, int G, int kind, const Cx<T>* cb, int ldc, T* rt, int ldr, Tables<T> tb) {
  // w in [0, G * N)
  const int g = w % G, k = w / G;
  const Cx<T> zk = cb[g * ldc + k];
  const Cx<T> zr = conj(cb[g * ldc + (k == 0 ? 0 : N - k)]);
  // V_a = (zk + zr)/2, V_b = (zk - zr)/(2i); y = 2 Re(quarter[k] V)
  const Cx<T> va = zk + zr;                    // 2 V_a
  const Cx<T> d = zk - zr;
  const Cx<T> vb = {d.y, -d.x};                // 2 V_b
  const Cx<T> qk = tb.quarter[k];
  const T ya = qk.x * va.x - qk.y * va.y;      // Re(q * 2V_a) = 2 Re(q V_a)
  const T yb = qk.x * vb.x - qk.y * vb.y;
  const int dst = (kind == O10) ? N - 1 - k : k;
  rt[(2 * g) * ldr + dst] = ya;
  rt[(2 * g + 1) * ldr + dst] = yb;
}

// (3) inverse kinds: two real coefficient pencils -> packed complex, conjugated
//     (the inverse DFT is run as conj(FFT(conj(.))))
template <typename T, int N>
QHD void inv_pack(int w, int G, int kind, const T* rt, int ldr, Cx<T>* cb, int ldc, Tables<T> tb) {
  // w in [0, G * N)
  const int g = w % G, k = w / G;
  const T* a = rt + (2 * g) * ldr;
  const T* b = rt + (2 * g + 1) * ldr;
  const bool rev = kind == O01;
  auto at = [&](const T* s, int i) -> T {   // y_i with y_N = 0, reversed for O01
    return i >= N ? T(0) : s[rev ? N - 1 - i : i];
  };
  const T ak = at(a, k), bk = at(b, k);
  const T an = k ? at(a, N - k) : T(0), bn = k ? at(b, N - k) : T(0);
  // V = e^{+i pi k/2N} (y_k - i y_{N-k});  packed = V_a + i V_b
  const Cx<T> e = conj(tb.quarter[k]);
  const Cx<T> va = cmul(e, Cx<T>{ak, -an});
  const Cx<T> vb = cmul(e, Cx<T>{bk, -bn});
  const Cx<T> z = {va.x - vb.y, va.y + vb.x};
  cb[g * ldc + k] = conj(z);
}

// (4) inverse kinds: conj(FFT) result -> two real pencils (Makhoul un-reorder)
template <typename T, int N>
QHD void inv_unpack(int w, int G, int kind, const Cx<T>* cb, int ldc, T* rt, int ldr) {
  // w in [0, G * N/2)
  const int g = w % G, t = w / G;
  const Cx<T> u0 = conj(cb[g * ldc + t]);
  const Cx<T> u1 = conj(cb[g * ldc + N - 1 - t]);
  const T sgn = (kind == O01) ? T(-1) : T(1);
  rt[(2 * g) * ldr + 2 * t] = u0.x;
  rt[(2 * g) * ldr + 2 * t + 1] = sgn * u1.x;
  rt[(2 * g + 1) * ldr + 2 * t] = u0.y;
  rt[(2 * g + 1) * ldr + 2 * t + 1] = sgn * u1.y;
}

// ---------------------------------------------------------------------------
// Whole tile: P = 2G real pencils of length N in buffer `a` (pencil stride
// LD = tile_ld(N) reals) are transformed with `kind`; `b` is a second buffer
// of the same size (G pencils of LD complex).  Returns the buffer that holds
// the result (a or b), real layout, stride LD.
// `ex.loop(count, f)` runs f(w) for w < count across the CTA and then
// synchronises (device), or serially (host unit test).
// ---------------------------------------------------------------------------
QHD constexpr int tile_ld(int n) { return n + 1; }

template <typename T, int N, class Exec>
QHD T* r2r_tile(Exec& ex, int kind, int G, T* a, T* b, Tables<T> tb) {
  constexpr RadixPlan plan = radix_plan(N);
  constexpr int LD = tile_ld(N);
  static_assert(plan.n_stages > 0, "unsupported transform length");
  Cx<T>* ca = reinterpret_cast<Cx<T>*>(a);
  Cx<T>* cbuf = reinterpret_cast<Cx<T>*>(b);
  if (is_forward(kind)) {
    ex.loop(G * (N / 2), [&](int w) { fwd_pack<T, N>(w, G, kind, a, LD, cbuf, LD); });
  } else {
    ex.loop(G * N, [&](int w) { inv_pack<T, N>(w, G, kind, a, LD, cbuf, LD, tb); });
  }
  Cx<T>* src = cbuf;
  Cx<T>* dst = ca;
  int n = N, s = 1;
#pragma unroll
  for (int st = 0; st < plan.n_stages; ++st) {
    const int r = plan.r[st];
    const int cnt = G * (N / r);
    if (r == 16) ex.loop(cnt, [&](int w) { stockham_stage<T, N, 16>(w, G, src, dst, n, s, LD, tb); });
    else if (r == 8) ex.loop(cnt, [&](int w) { stockham_stage<T, N, 8>(w, G, src, dst, n, s, LD, tb); });
    else if (r == 4) ex.loop(cnt, [&](int w) { stockham_stage<T, N, 4>(w, G, src, dst, n, s, LD, tb); });
    else if (r == 3) ex.loop(cnt, [&](int w) { stockham_stage<T, N, 3>(w, G, src, dst, n, s, LD, tb); });
    else ex.loop(cnt, [&](int w) { stockham_stage<T, N, 2>(w, G, src, dst, n, s, LD, tb); });
    n /= r;
    s *= r;
    Cx<T>* t = src; src = dst; dst = t;
  }
  // spectrum is in `src`; unpack into the other buffer
  T* out = reinterpret_cast<T*>(dst);
  if (is_forward(kind)) {
    ex.loop(G * N, [&](int w) { fwd_unpack<T, N>(w, G, kind, src, LD, out, LD, tb); });
  } else {
    ex.loop(G * (N / 2), [&](int w) { inv_unpack<T, N>(w, G, kind, src, LD, out, LD); });
  }
  return out;
}

}  // namespace quasi
