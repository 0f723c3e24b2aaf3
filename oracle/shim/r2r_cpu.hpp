// CPU restatement of FFTW's real-to-real kinds REDFT10 / REDFT01 / RODFT10 /
// RODFT01 (unnormalised, FFTW 3.3 manual section "Real even/odd DFTs").
//
// TEST INFRASTRUCTURE ONLY: used by oracle/shim to let the reference's own
// quasi.cpp run without FFTW.  Never linked into libquasi_gpu.so.
//
// Definitions (n = 0..N-1, k = 0..N-1):
//   REDFT10  y_k = 2 sum_n x_n cos(pi k (2n+1) / 2N)
//   REDFT01  y_k = x_0 + 2 sum_{n>=1} x_n cos(pi n (2k+1) / 2N)
//   RODFT10  y_k = 2 sum_n x_n sin(pi (k+1)(2n+1) / 2N)
//   RODFT01  y_k = (-1)^k x_{N-1} + 2 sum_{n<N-1} x_n sin(pi (n+1)(2k+1) / 2N)
// Algorithm: Makhoul (1980) reordering + one complex FFT per PAIR of real
// sequences (real and imaginary parts), mixed-radix (4, 3, 2) Stockham.
// RODFT10(x)_k = REDFT10((-1)^n x_n)_{N-1-k};  RODFT01(x)_k = (-1)^k REDFT01(rev x)_k.
#pragma once
#include <cmath>
#include <complex>
#include <stdexcept>
#include <vector>

namespace quasi_cpu {

using cplx = std::complex<double>;

enum Kind { REDFT10 = 0, REDFT01 = 1, RODFT10 = 2, RODFT01 = 3 };

class R2R1D {
 public:
  explicit R2R1D(int n) : n_(n) {
    if (n < 2 || (n & 1)) throw std::invalid_argument("r2r length must be even and >= 2");
    int m = n;
    while (m > 1) {
      if (m % 4 == 0) { radix_.push_back(4); m /= 4; }
      else if (m % 2 == 0) { radix_.push_back(2); m /= 2; }
      else if (m % 3 == 0) { radix_.push_back(3); m /= 3; }
      else throw std::invalid_argument("r2r length must be 2^a 3^b");
    }
    root_.resize(n);
    for (int t = 0; t < n; ++t) {
      long double a = -2.0L * 3.14159265358979323846264338327950288L * t / n;
      root_[t] = cplx((double)std::cos(a), (double)std::sin(a));
    }
    quarter_.resize(n);
    for (int t = 0; t < n; ++t) {
      long double a = -3.14159265358979323846264338327950288L * t / (2.0L * n);
      quarter_[t] = cplx((double)std::cos(a), (double)std::sin(a));
    }
  }

  int size() const { return n_; }

  // Transform two real sequences a and b (stride 1, length N) in place.
  // b may be null (a single sequence).
  void pair(Kind kind, double* a, double* b, std::vector<cplx>& w1, std::vector<cplx>& w2) const {
    const int N = n_;
    w1.resize(N); w2.resize(N);
    if (kind == REDFT10 || kind == RODFT10) {
      const bool odd = kind == RODFT10;
      for (int t = 0; t < N / 2; ++t) {
        double sa0 = a[2 * t], sa1 = a[2 * t + 1];
        double sb0 = b ? b[2 * t] : 0.0, sb1 = b ? b[2 * t + 1] : 0.0;
        if (odd) { sa1 = -sa1; sb1 = -sb1; }   // (-1)^n x_n, 2t even, 2t+1 odd
        w1[t] = cplx(sa0, sb0);
        w1[N - 1 - t] = cplx(sa1, sb1);
      }
      fft(w1, w2);
      for (int k = 0; k < N; ++k) {
        cplx zk = w1[k], zr = std::conj(w1[(N - k) % N]);
        cplx va = 0.5 * (zk + zr), vb = cplx(0, -0.5) * (zk - zr);
        double ya = 2.0 * (quarter_[k] * va).real();
        double yb = 2.0 * (quarter_[k] * vb).real();
        int dst = odd ? N - 1 - k : k;
        w2[dst] = cplx(ya, yb);
      }
      for (int k = 0; k < N; ++k) { a[k] = w2[k].real(); if (b) b[k] = w2[k].imag(); }
    } else {
      const bool odd = kind == RODFT01;
      // input y (DCT-II coefficients); for RODFT01 reverse the input first
      auto ya = [&](int k) { return k >= N ? 0.0 : (odd ? a[N - 1 - k] : a[k]); };
      auto yb = [&](int k) { return (k >= N || !b) ? 0.0 : (odd ? b[N - 1 - k] : b[k]); };
      for (int k = 0; k < N; ++k) {
        cplx e = std::conj(quarter_[k]);   // exp(+i pi k / 2N)
        cplx Va = e * cplx(ya(k), -ya(N - k == N ? N : N - k));
        cplx Vb = e * cplx(yb(k), -yb(N - k == N ? N : N - k));
        // k = 0: x_N := 0
        if (k == 0) { Va = cplx(ya(0), 0.0); Vb = cplx(yb(0), 0.0); }
        w1[k] = Va + cplx(0, 1) * Vb;
      }
      // unnormalised inverse DFT = conj(FFT(conj(.)))
      for (int k = 0; k < N; ++k) w1[k] = std::conj(w1[k]);
      fft(w1, w2);
      for (int k = 0; k < N; ++k) w1[k] = std::conj(w1[k]);
      for (int t = 0; t < N / 2; ++t) {
        cplx u0 = w1[t], u1 = w1[N - 1 - t];
        double s = 1.0;
        double a0 = u0.real(), a1 = u1.real(), b0 = u0.imag(), b1 = u1.imag();
        if (odd) { s = -1.0; }
        a[2 * t] = a0; a[2 * t + 1] = s * a1;
        if (b) { b[2 * t] = b0; b[2 * t + 1] = s * b1; }
      }
    }
  }

 private:
  // forward complex DFT (exp(-2 pi i nk/N)) in place, Stockham DIF, work = scratch
  void fft(std::vector<cplx>& x, std::vector<cplx>& work) const {
    const int N = n_;
    cplx* src = x.data();
    cplx* dst = work.data();
    int s = 1;   // stride of the already-split subsequences
    int n = N;   // current sub-transform length
    for (int r : radix_) {
      const int m = n / r;
      for (int p = 0; p < m; ++p) {
        for (int q = 0; q < s; ++q) {
          cplx a[4];
          for (int t = 0; t < r; ++t) a[t] = src[q + s * (p + t * m)];
          cplx out[4];
          if (r == 2) {
            out[0] = a[0] + a[1];
            out[1] = a[0] - a[1];
          } else if (r == 4) {
            cplx t0 = a[0] + a[2], t1 = a[0] - a[2], t2 = a[1] + a[3], t3 = a[1] - a[3];
            cplx mit3(t3.imag(), -t3.real());   // -i * t3
            out[0] = t0 + t2; out[2] = t0 - t2;
            out[1] = t1 + mit3; out[3] = t1 - mit3;
          } else {   // r == 3
            const double c = -0.5, sn = 0.86602540378443864676372317075294;
            cplx t1 = a[1] + a[2], t2 = a[1] - a[2];
            out[0] = a[0] + t1;
            cplx base = a[0] + c * t1;
            cplx rot(sn * t2.imag(), -sn * t2.real());   // -i sin(2pi/3) t2
            out[1] = base + rot;
            out[2] = base - rot;
          }
          // twiddle W_n^{p u} = root_[(N/n) * p * u]
          for (int u = 0; u < r; ++u) {
            int e = (int)(((long long)(N / n) * p * u) % N);
            dst[q + s * (r * p + u)] = out[u] * root_[e];
          }
        }
      }
      std::swap(src, dst);
      s *= r;
      n = m;
    }
    if (src != x.data()) for (int t = 0; t < N; ++t) x[t] = src[t];
  }

  int n_;
  std::vector<int> radix_;
  std::vector<cplx> root_, quarter_;
};

}  // namespace quasi_cpu
