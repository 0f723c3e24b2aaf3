// Host-side check of the tensor-core pass's data layout and arithmetic: the
// swizzled operand offsets of tc_pass.cuh (A: K-major, B: MN-major, 128-byte
// swizzle) are bijections inside their buffers; every (pair, chunk) of a tile
// is loaded by exactly one thread and every output row written by exactly one
// lane; and the folded split-BF16 contraction, computed here from the swizzled
// images exactly as the kernel addresses them (B converted with the same
// round-to-nearest BF16 split), reproduces FFTW's REDFT10/01, RODFT10/01 in
// long double.  Prints "layout ok" lines and the worst relative error per kind.
#include <cmath>
#include <cstdio>
#include <random>
#include <set>
#include <vector>

#include "../../smaiso_quasi_b200/csrc/tc_pass.cuh"

using namespace quasi;
using namespace quasi::tc;

static long double coef(int kind, int N, int k, int n) {
  const long double PI = 3.141592653589793238462643383279502884L;
  if (kind == E10) return 2 * cosl(PI * k * (2 * n + 1) / (2 * N));
  if (kind == E01) return (n == 0) ? 1 : 2 * cosl(PI * n * (2 * k + 1) / (2 * N));
  if (kind == O10) return 2 * sinl(PI * (k + 1) * (2 * n + 1) / (2 * N));
  return (n == N - 1) ? ((k % 2) ? -1 : 1) : 2 * sinl(PI * (n + 1) * (2 * k + 1) / (2 * N));
}

static float bf(float x) { return bf16_value(bf16_bits(x)); }

int main() {
  // offsets: bijective and in bounds
  std::set<int> sa, sb;
  for (int r = 0; r < kH; ++r)
    for (int k = 0; k < kH; ++k) {
      const int o = a_offset(r, k);
      if (o < 0 || o + 2 > kMat || o % 2) { printf("a_offset out of range\n"); return 1; }
      sa.insert(o);
    }
  for (int k = 0; k < kH; ++k)
    for (int n = 0; n < kCols; ++n) {
      const int o = b_offset(k, n);
      if (o < 0 || o + 2 > kBMat || o % 2) { printf("b_offset out of range\n"); return 1; }
      sb.insert(o);
    }
  printf("layout a %d %zu\nlayout b %d %zu\n", kH * kH, sa.size(), kH * kCols, sb.size());
  // the load mapping: pair P = tid + 256 r -> (m = P >> 4, q = P & 15) covers every (m, q) once
  std::set<int> pairs;
  for (int tid = 0; tid < kThreads; ++tid)
    for (int r = 0; r < (kH * kCols / 4) / kThreads; ++r) pairs.insert(tid + kThreads * r);
  printf("layout pairs %d %zu\n", kH * (kCols / 4), pairs.size());
  // epilogue: (warp, lane) -> rows; both directions cover 0..255 once per column half
  for (int fwd = 0; fwd < 2; ++fwd) {
    std::set<int> rows[2];
    for (int warp = 0; warp < 8; ++warp)
      for (int lane = 0; lane < 32; ++lane) {
        const int sp = warp & 3, ch = warp >> 2, p = sp * 32 + lane;
        rows[ch].insert(fwd ? 2 * p : p);
        rows[ch].insert(fwd ? 2 * p + 1 : kN - 1 - p);
      }
    printf("layout rows%d %d %zu %zu\n", fwd, kN, rows[0].size(), rows[1].size());
  }
  // arithmetic, from the swizzled images
  std::mt19937_64 rng(5);
  std::normal_distribution<double> nd;
  std::vector<float> x(kN * kCols);
  for (auto& v : x) v = float(nd(rng));
  for (int kind = 0; kind < 4; ++kind) {
    const std::vector<uint16_t> img = folded_matrices(kind);
    auto A = [&](int mat, int part, int p, int m) {   // mat 0 even / 1 odd, part 0 hi / 1 lo
      return bf16_value(img[(mat * 2 * kMat + part * kMat + a_offset(p, m)) / 2]);
    };
    const bool fwd = is_forward(kind);
    std::vector<uint16_t> bimg(kSmemB / 2);
    for (int m = 0; m < kH; ++m)
      for (int n = 0; n < kCols; ++n) {
        const float a = x[(fwd ? m : 2 * m) * kCols + n], b = x[(fwd ? kN - 1 - m : 2 * m + 1) * kCols + n];
        const float s = fwd ? a + b : a, d = fwd ? a - b : b;
        const float v[2] = {s, d};
        for (int mat = 0; mat < 2; ++mat) {
          const uint16_t hi = bf16_bits(v[mat]);
          const uint16_t lo = bf16_bits(v[mat] - bf16_value(hi));
          bimg[(mat * 2 * kBMat + b_offset(m, n)) / 2] = hi;
          bimg[(mat * 2 * kBMat + kBMat + b_offset(m, n)) / 2] = lo;
        }
      }
    auto B = [&](int mat, int part, int m, int n) {
      return bf16_value(bimg[(mat * 2 * kBMat + part * kBMat + b_offset(m, n)) / 2]);
    };
    double num = 0, den = 0;
    for (int n = 0; n < kCols; ++n) {
      std::vector<double> y(kN);
      for (int p = 0; p < kH; ++p) {
        double D[2];
        for (int mat = 0; mat < 2; ++mat) {
          float acc = 0;   // FP32 accumulation of the three products
          for (int m = 0; m < kH; ++m)
            acc += A(mat, 0, p, m) * B(mat, 1, m, n) + A(mat, 1, p, m) * B(mat, 0, m, n) +
                   A(mat, 0, p, m) * B(mat, 0, m, n);
          D[mat] = acc;
        }
        if (fwd) { y[2 * p] = D[0]; y[2 * p + 1] = D[1]; }
        else { y[p] = float(D[0] + D[1]); y[kN - 1 - p] = float(D[0] - D[1]); }
      }
      for (int k = 0; k < kN; ++k) {
        long double ex = 0;
        for (int j = 0; j < kN; ++j) ex += coef(kind, kN, k, j) * (long double)x[j * kCols + n];
        num += double((y[k] - ex) * (y[k] - ex));
        den += double(ex * ex);
      }
    }
    printf("kind %d %.3e\n", kind, std::sqrt(num / den));
  }
  return 0;
}
