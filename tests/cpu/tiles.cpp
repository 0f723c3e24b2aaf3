// Host-side check of the tile transforms' indexing: the exact device code of
// r2r_core.cuh (pencil-major tiles of the x / y passes, in place and out of
// place) and z_pass.cuh (the element-fastest tile of the z pass, with and
// without the one-row shift) run serially, every "thread" of a phase reading
// before any writes, as the kernels' barriers order them.  Each result is
// compared with FFTW's unnormalised REDFT10/01, RODFT10/01 definitions in long
// double; prints the worst relative error per (type, length).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../smaiso_quasi_b200/csrc/z_pass.cuh"

using namespace quasi;

template <int NT> struct HostExec {
  template <class R, class W, class Regs> void phase(R rd, W wr, int, Regs&, bool, bool) {
    std::vector<Regs> regs(NT);
    for (int t = 0; t < NT; ++t) rd(t, regs[t]);
    for (int t = 0; t < NT; ++t) wr(t, regs[t]);
  }
  void sync() {}
};

template <typename T> struct HSrc {
  const T* a; int ld;
  void pair(int g, int n, T& x, T& y) const { x = a[(2 * g) * ld + n]; y = a[(2 * g + 1) * ld + n]; }
};
template <typename T> struct HSnk {
  T* a; int ld;
  void put(int g, int n, T x, T y) const { a[(2 * g) * ld + n] = x; a[(2 * g + 1) * ld + n] = y; }
};

static long double coef(int kind, int N, int k, int n) {
  const long double PI = 3.141592653589793238462643383279502884L;
  if (kind == 0) return 2 * cosl(PI * k * (2 * n + 1) / (2 * N));
  if (kind == 1) return (n == 0) ? 1 : 2 * cosl(PI * n * (2 * k + 1) / (2 * N));
  if (kind == 2) return 2 * sinl(PI * (k + 1) * (2 * n + 1) / (2 * N));
  return (n == N - 1) ? ((k % 2) ? -1 : 1) : 2 * sinl(PI * (n + 1) * (2 * k + 1) / (2 * N));
}

template <typename T> struct Tabs {
  std::vector<Cx<T>> root, quarter;
  explicit Tabs(int N) : root(N), quarter(N) {
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int t = 0; t < N; t++) {
      root[t] = {(T)cosl(-2 * PI * t / N), (T)sinl(-2 * PI * t / N)};
      quarter[t] = {(T)cosl(-PI * t / (2 * N)), (T)sinl(-PI * t / (2 * N))};
    }
  }
  Tables<T> get() const { return Tables<T>{root.data(), quarter.data()}; }
};

// worst |out - exact| / max|exact| over the P pencils; x[p][n], out[p][k] at stride ld
template <typename T>
double worst(int kind, int N, int P, const std::vector<T>& x, int xld, const T* out, int old, int ks) {
  double w = 0, mx = 0;
  for (int p = 0; p < P; p++)
    for (int k = 0; k < N; k++) {
      long double s = 0;
      for (int n = 0; n < N; n++) {
        const long double v = n + ks < N ? (long double)x[p * xld + n + ks] : 0.0L;
        s += coef(kind, N, k, n) * v;
      }
      w = std::max(w, (double)fabsl(out[p * old + k] - s));
      mx = std::max(mx, (double)fabsl(s));
    }
  return w / mx;
}

template <typename T, int N, int G, int NT> double tile_case(int kind, bool inplace) {
  std::mt19937_64 rng(N * 7 + kind);
  std::uniform_real_distribution<double> U(-1, 1);
  Tabs<T> tb(N);
  const int P = 2 * G, LD = tile_ld(N);
  std::vector<T> A(P * LD, T(0)), Y(P * LD, T(0));
  for (int p = 0; p < P; p++)
    for (int n = 0; n < N; n++) A[p * LD + n] = (T)U(rng);
  const std::vector<T> X = A;
  HostExec<NT> ex;
  if (inplace) {
    r2r_tile_inplace<T, N, G, NT>(ex, 0, kind, A.data(), tb.get());
    return worst(kind, N, P, X, LD, A.data(), LD, 0);
  }
  std::vector<Cx<T>> cb(G * LD);
  r2r_tile<T, N, G, NT, false>(ex, 0, kind, cb.data(), HSrc<T>{X.data(), LD}, HSnk<T>{Y.data(), LD}, tb.get());
  return worst(kind, N, P, X, LD, Y.data(), LD, 0);
}

template <typename T, int N, int G, int NT, int SUB = 1> double ztile_case(int kind, int ks) {
  using Z = ZTile<T, N, G, NT, SUB>;
  std::mt19937_64 rng(N * 11 + kind);
  std::uniform_real_distribution<double> U(-1, 1);
  Tabs<T> tb(N);
  const int P = 2 * G;
  std::vector<T> raw(P * N);
  for (auto& v : raw) v = (T)U(rng);
  std::vector<Cx<T>> cb(Z::cb_bytes() / sizeof(Cx<T>), Cx<T>{T(1e30), T(1e30)});
  T* stg = reinterpret_cast<T*>(cb.data());
  std::vector<typename Z::template Regs<Z::R1>> r1(NT);
  for (int t = 0; t < NT; ++t) Z::first_read(t, typename Z::Rows{raw.data(), ks}, kind, tb.get(), r1[t]);
  for (int t = 0; t < NT; ++t) Z::template stage_write<Z::R1, 1>(t, cb.data(), r1[t]);
  HostExec<NT> ex;
  ztile_after_first<T, N, G, NT, SUB>(ex, 0, kind, cb.data(), stg, tb.get());
  // rows as [p][n] whatever the block layout
  std::vector<T> xd(P * N), od(P * N);
  for (int p = 0; p < P; ++p)
    for (int n = 0; n < N; ++n) {
      xd[p * N + n] = raw[Z::ri(p, n)];
      od[p * N + n] = stg[Z::ri(p, n)];
    }
  return worst(kind, N, P, xd, N, od.data(), N, ks);
}

template <typename T, int N, int G, int NT> void tiles() {
  double w = 0;
  for (int k = 0; k < 4; k++) w = std::max({w, tile_case<T, N, G, NT>(k, true), tile_case<T, N, G, NT>(k, false)});
  printf("tile %s %d %.3g\n", sizeof(T) == 8 ? "f64" : "f32", N, w);
}
template <typename T, int N, int G, int SUB = 1> void ztiles() {
  double w = 0;
  for (int k = 0; k < 4; k++)
    w = std::max({w, ztile_case<T, N, G, 256, SUB>(k, 0), ztile_case<T, N, G, 256, SUB>(k, 1)});
  printf("ztile %s %d %.3g\n", sizeof(T) == 8 ? "f64" : "f32", N * 10 + SUB, w);
}

// the warp tiles of the x / y passes: one warp (32 threads) on 2 float or 1 double pencils
template <typename T, int N> void wtiles() {
  constexpr int G = sizeof(T) == 4 ? 2 : 1;
  double w = 0;
  for (int k = 0; k < 4; k++) w = std::max({w, tile_case<T, N, G, 32>(k, true), tile_case<T, N, G, 32>(k, false)});
  printf("wtile %s %d %.3g\n", sizeof(T) == 8 ? "f64" : "f32", N, w);
}

// the warp tiles of the z pass: one warp (32 threads) on 2 float or 1 double pencils
template <typename T, int N> void zwtiles() {
  constexpr int G = sizeof(T) == 4 ? 2 : 1;
  double w = 0;
  for (int k = 0; k < 4; k++) w = std::max({w, ztile_case<T, N, G, 32>(k, 0), ztile_case<T, N, G, 32>(k, 1)});
  printf("zwtile %s %d %.3g\n", sizeof(T) == 8 ? "f64" : "f32", N, w);
}

int main() {
  tiles<double, 8, 8, 128>(); tiles<double, 16, 8, 256>(); tiles<double, 32, 8, 128>(); tiles<double, 64, 8, 256>();
  tiles<double, 96, 8, 256>(); tiles<double, 128, 8, 256>(); tiles<double, 192, 8, 256>(); tiles<double, 256, 8, 256>();
  tiles<double, 512, 4, 256>(); tiles<float, 256, 16, 256>(); tiles<float, 96, 16, 256>(); tiles<float, 512, 8, 256>();
  ztiles<double, 16, 8>(); ztiles<double, 32, 8>(); ztiles<double, 64, 8>(); ztiles<double, 96, 8>();
  ztiles<double, 128, 8>(); ztiles<double, 192, 8>(); ztiles<double, 256, 8>(); ztiles<double, 8, 8>();
  ztiles<float, 16, 16>(); ztiles<float, 64, 16>(); ztiles<float, 96, 16>(); ztiles<float, 128, 16>();
  ztiles<float, 192, 16>(); ztiles<float, 256, 16>();
  ztiles<double, 512, 4, 2>(); ztiles<float, 512, 8, 2>();   // two 256-element blocks per row
  // the warp tiles of the x / y passes: one warp on 2 float or 1 double pencils
  wtiles<double, 64>(); wtiles<double, 96>(); wtiles<double, 128>(); wtiles<double, 192>(); wtiles<double, 256>();
  wtiles<float, 64>(); wtiles<float, 128>(); wtiles<float, 256>();
  zwtiles<double, 64>(); zwtiles<double, 96>(); zwtiles<double, 128>(); zwtiles<double, 192>(); zwtiles<double, 256>();
  zwtiles<float, 64>(); zwtiles<float, 96>(); zwtiles<float, 128>(); zwtiles<float, 192>(); zwtiles<float, 256>();
  return 0;
}
