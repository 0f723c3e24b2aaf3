// The z pass (transform along the contiguous axis) as a persistent TMA
// kernel that never touches global memory from its threads:
//
//   TMA load of P = 2G dense rows [p][n]  ->  element-fastest tile FFT
//   (first stage reads the dense rows, later stages a padded complex tile)
//   ->  dense staging rows [p][n]  ->  TMA store.
//
// Element-fastest: the work items of a stage are numbered butterfly-fastest
// within a pencil (g = w / (N/R)), so a warp reads and writes runs of one
// row.  Where two pencils share a warp, odd pencils take the partner half of
// each (even n, odd n) or (e, e + N/R) pair first, which puts the two
// half-warps on disjoint banks.  The padded tile keeps complex e of pencil g
// at g * LDC + e + e / R1 (R1 = first radix), conflict-free for the stage-1
// writes (stride R1) and every later stage.
//
// Kinds, Makhoul reordering and the pairing of two real pencils into one
// complex DFT are those of r2r_core.cuh (FFTW's REDFT10/01, RODFT10/01).
#pragma once
#ifdef __CUDACC__
#include "r2r_pass.cuh"
#else
#include <cstddef>

#include "r2r_core.cuh"   // the tile transform alone (host-side tests)
#endif

namespace quasi {

// SUB: the dense rows are held as SUB blocks [SUB][2G][N/SUB] (a TMA box side
// is at most 256 elements, so N = 512 moves as two boxes per row).
template <typename T, int N, int G, int NT, int SUB = 1>
struct ZTile {
  static constexpr RadixPlan plan = radix_plan(N, max_radix<T>());
  static constexpr int BN = N / SUB;
  static_assert(BN * SUB == N, "SUB divides N");
  // element n of dense row r
  QHD static constexpr int ri(int r, int n) {
    return SUB == 1 ? r * N + n : (n / BN) * (2 * G * BN) + r * BN + (n - (n / BN) * BN);
  }
  static_assert(plan.n_stages > 0, "unsupported transform length");
  static constexpr int R1 = plan.r[0];
  QHD static constexpr int phi(int e) { return e + e / R1; }
  // padded pencil stride (complex).  FP32: rounded to 8 mod 16 so that two
  // pencils sharing a warp start on different bank halves; FP64 (a warp
  // never spans two pencils of the sizes that matter) just even
  static constexpr int LDC =
      sizeof(T) == 8 ? ((phi(N - 1) + 2) / 2) * 2 : ((phi(N - 1) + 1 + 7) / 16) * 16 + 8;
  static constexpr size_t cb_bytes() { return size_t(G) * LDC * sizeof(Cx<T>); }
  static_assert(LDC >= N, "the staging rows overlay the padded tile");

  template <int R> static constexpr int per_thread() { return (G * (N / R) + NT - 1) / NT; }
  template <int R> struct Regs { Cx<T> v[per_thread<R>()][R]; };

  // stage-1 input e of pencil g from the dense rows (row[n + ks], zero past
  // the end): forward kinds with the Makhoul reorder, inverse kinds with the
  // pre-twiddle of r2r_core's first_input
  struct Rows {
    const T* raw;
    int ks;
    QHD T at(int r, int n) const { return n + ks < N ? raw[ri(r, n + ks)] : T(0); }
  };
  // the same with the shift fixed at compile time (the kernel's form); KS = 2:
  // row[n + 1] times -mk[n] (a z gradient's shift and wavenumber, zero at the top)
  template <int KS> struct RowsK {
    const T* raw;
    const T* mk = nullptr;
    QHD T at(int r, int n) const {
      if constexpr (KS == 0) return raw[ri(r, n)];
      else if constexpr (KS == 1) return n + 1 < N ? raw[ri(r, n + 1)] : T(0);
      else return n + 1 < N ? -mk[n] * raw[ri(r, n + 1)] : T(0);
    }
  };
  template <class Src>
  QHD static Cx<T> fwd_in(const Src& src, int kind, int g, int e) {
    int n;
    T sgn = T(1);
    if (e < N / 2) n = 2 * e;
    else { n = 2 * (N - 1 - e) + 1; if (kind == O10) sgn = T(-1); }
    return Cx<T>{sgn * src.at(2 * g, n), sgn * src.at(2 * g + 1, n)};
  }
  template <class Src>
  QHD static Cx<T> inv_in(const Src& src, int kind, int g, int k, Tables<T> tb) {
    const bool rev = kind == O01;
    const int n0 = rev ? N - 1 - k : k;
    const T ak = src.at(2 * g, n0), bk = src.at(2 * g + 1, n0);
    T an = T(0), bn = T(0);
    if (k) {
      const int n1 = rev ? k - 1 : N - k;
      an = src.at(2 * g, n1);
      bn = src.at(2 * g + 1, n1);
    }
    const Cx<T> q = tb.quarter[k];
    const Cx<T> ec = {q.x, -q.y};
    const Cx<T> va = cmul(ec, Cx<T>{ak, -an});
    const Cx<T> vb = cmul(ec, Cx<T>{bk, -bn});
    return Cx<T>{va.x - vb.y, -(va.y + vb.x)};
  }

  // first stage read (s = 1): butterfly b of pencil g takes e = b + t N/R
  // tw1 (optional): the first stage's twiddles W_N^{b u} as tw1[u * (N/R1) + b]
  // (a warp reads consecutive entries); otherwise tb.root[b u]
  template <class Src>
  QHD static void first_read(int tid, const Src& src, int kind, Tables<T> tb, Regs<R1>& r,
                             const Cx<T>* tw1 = nullptr) {
    constexpr int R = R1, M = N / R;
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * M) break;
      const int g = w / M, b = w - g * M;
      const bool x = g & 1;
      if (is_forward(kind)) {
        // pairs (t, t + R/2): even and odd Makhoul positions
#pragma unroll
        for (int t = 0; t < R / 2; ++t) {
          const Cx<T> A = fwd_in(src, kind, g, b + M * (x ? t + R / 2 : t));
          const Cx<T> B = fwd_in(src, kind, g, b + M * (x ? t : t + R / 2));
          r.v[c][t] = x ? B : A;
          r.v[c][t + R / 2] = x ? A : B;
        }
      } else {
        // pairs (t, t ^ 1): elements M apart
#pragma unroll
        for (int t = 0; t < R; t += 2) {
          const Cx<T> A = inv_in(src, kind, g, b + M * (x ? t + 1 : t), tb);
          const Cx<T> B = inv_in(src, kind, g, b + M * (x ? t : t + 1), tb);
          r.v[c][t] = x ? B : A;
          r.v[c][t + 1] = x ? A : B;
        }
      }
      Dft<T, R>::run(r.v[c]);
#pragma unroll
      for (int u = 1; u < R; ++u)
        if (b) r.v[c][u] = cmul(r.v[c][u], tw1 ? tw1[u * M + b] : tb.root[b * u]);
    }
  }

  // stage ST > 0 read from the padded tile (stride s, sub-length n = N / s)
  template <int R, int n, int s>
  QHD static void stage_read(int tid, const Cx<T>* cb, Tables<T> tb, Regs<R>& r) {
    constexpr int m = n / R, NB = N / R;
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * NB) break;
      const int g = w / NB, bfl = w - g * NB;
      const int p = bfl / s, q = bfl - p * s;
#pragma unroll
      for (int t = 0; t < R; ++t) r.v[c][t] = cb[g * LDC + phi(q + s * (p + t * m))];
      Dft<T, R>::run(r.v[c]);
      const int step = (N / n) * p;
#pragma unroll
      for (int u = 1; u < R; ++u)
        if (p) r.v[c][u] = cmul(r.v[c][u], tb.root[step * u]);
    }
  }

  // stage write into the padded tile
  template <int R, int s>
  QHD static void stage_write(int tid, Cx<T>* cb, const Regs<R>& r) {
    constexpr int NB = N / R;
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * NB) break;
      const int g = w / NB, bfl = w - g * NB;
      const int p = bfl / s, q = bfl - p * s;
#pragma unroll
      for (int u = 0; u < R; ++u) cb[g * LDC + phi(q + s * (R * p + u))] = r.v[c][u];
    }
  }

  // last stage of an inverse kind: u_k = conj(F_k) -> x_{2k} (k < N/2) or
  // x_{2(N-1-k)+1}, into the dense staging rows (real pencil 2g, 2g + 1)
  QHD static void put_inv(T* stg, int kind, int g, int k, Cx<T> f) {
    int n;
    T sgn = T(1);
    if (k < N / 2) n = 2 * k;
    else { n = 2 * (N - 1 - k) + 1; if (kind == O01) sgn = T(-1); }
    stg[ri(2 * g, n)] = sgn * f.x;
    stg[ri(2 * g + 1, n)] = -sgn * f.y;
  }
  template <int R, int s>
  QHD static void last_write_inv(int tid, T* stg, int kind, const Regs<R>& r) {
    constexpr int NB = N / R;   // = s: the last stage has p = 0
#pragma unroll
    for (int c = 0; c < per_thread<R>(); ++c) {
      const int w = tid + c * NT;
      if (w >= G * NB) break;
      const int g = w / NB, q = w - g * NB;
      const bool x = g & 1;
      if constexpr (R % 2 == 0) {
        // pairs (u, u + R/2): even and odd output positions
#pragma unroll
        for (int u = 0; u < R / 2; ++u) {
          const int ua = x ? u + R / 2 : u, ub = x ? u : u + R / 2;
          put_inv(stg, kind, g, q + s * ua, x ? r.v[c][u + R / 2] : r.v[c][u]);
          put_inv(stg, kind, g, q + s * ub, x ? r.v[c][u] : r.v[c][u + R / 2]);
        }
      } else {
#pragma unroll
        for (int u = 0; u < R; ++u) put_inv(stg, kind, g, q + s * u, r.v[c][u]);
      }
    }
  }

  // forward kinds: y(k), y(N-k) from (Z_k, Z_{N-k}); item k = 0 also makes
  // the self-paired y(N/2)
  static constexpr int kUnpack = (G * (N / 2) + NT - 1) / NT;
  struct UnpackRegs {
    T ya[kUnpack][2], yb[kUnpack][2];   // [1]: y(N-k), or y(N/2) for k = 0
  };
  QHD static void unpack_one(Cx<T> zk, Cx<T> zr_conj_src, Cx<T> qk, T& ya, T& yb) {
    const Cx<T> zr = conj(zr_conj_src);
    const Cx<T> va = zk + zr;
    const Cx<T> d = zk - zr;
    const Cx<T> vb = {d.y, -d.x};
    ya = qk.x * va.x - qk.y * va.y;
    yb = qk.x * vb.x - qk.y * vb.y;
  }
  QHD static void unpack_read(int tid, const Cx<T>* cb, Tables<T> tb, UnpackRegs& r) {
    constexpr int H = N / 2;
#pragma unroll
    for (int c = 0; c < kUnpack; ++c) {
      const int w = tid + c * NT;
      if (w >= G * H) break;
      const int g = w / H, k = w - g * H;
      const Cx<T>* pc = cb + g * LDC;
      const Cx<T> z0 = pc[phi(k)];
      const Cx<T> z1 = pc[phi(k ? N - k : H)];
      if (k) {
        unpack_one(z0, z1, tb.quarter[k], r.ya[c][0], r.yb[c][0]);
        unpack_one(z1, z0, tb.quarter[N - k], r.ya[c][1], r.yb[c][1]);
      } else {
        unpack_one(z0, z0, tb.quarter[0], r.ya[c][0], r.yb[c][0]);
        unpack_one(z1, z1, tb.quarter[H], r.ya[c][1], r.yb[c][1]);   // z1 = Z_{N/2}
      }
    }
  }
  QHD static void unpack_write(int tid, T* stg, int kind, const UnpackRegs& r) {
    constexpr int H = N / 2;
#pragma unroll
    for (int c = 0; c < kUnpack; ++c) {
      const int w = tid + c * NT;
      if (w >= G * H) break;
      const int g = w / H, k = w - g * H;
      auto idx = [&](int kk) { return kind == O10 ? N - 1 - kk : kk; };
      stg[ri(2 * g, idx(k))] = r.ya[c][0];
      stg[ri(2 * g + 1, idx(k))] = r.yb[c][0];
      const int k1 = k ? N - k : H;
      stg[ri(2 * g, idx(k1))] = r.ya[c][1];
      stg[ri(2 * g + 1, idx(k1))] = r.yb[c][1];
    }
  }
};

// Stages 1 .. last of the tile after the first stage's writes, then (forward)
// the unpack: `ex.phase(rd, wr, ...)` as in r2r_core.cuh.  Leaves the dense
// output rows in `stg` (which overlays `cb`) without a closing barrier: the
// caller fences them for the TMA store and synchronises.
template <typename T, int N, int G, int NT, int ST, int SUB = 1, class Exec>
QHD void ztile_rest(Exec& ex, int tid, int kind, Cx<T>* cb, T* stg, Tables<T> tb) {
  using Z = ZTile<T, N, G, NT, SUB>;
  if constexpr (ST < Z::plan.n_stages) {
    constexpr int R = Z::plan.r[ST];
    constexpr int s = stage_stride(N, ST, max_radix<T>()), n = N / s;
    constexpr bool last = ST == Z::plan.n_stages - 1;
    using Regs = typename Z::template Regs<R>;
    Regs regs;
    if (last && !is_forward(kind)) {
      ex.phase([&](int t, Regs& rg) { Z::template stage_read<R, n, s>(t, cb, tb, rg); },
               [&](int t, Regs& rg) { Z::template last_write_inv<R, s>(t, stg, kind, rg); }, tid, regs, true, false);
      return;
    }
    ex.phase([&](int t, Regs& rg) { Z::template stage_read<R, n, s>(t, cb, tb, rg); },
             [&](int t, Regs& rg) { Z::template stage_write<R, s>(t, cb, rg); }, tid, regs, true, true);
    if constexpr (last) {
      typename Z::UnpackRegs ur;
      ex.phase([&](int t, typename Z::UnpackRegs& rg) { Z::unpack_read(t, cb, tb, rg); },
               [&](int t, typename Z::UnpackRegs& rg) { Z::unpack_write(t, stg, kind, rg); }, tid, ur, true, false);
    } else {
      ztile_rest<T, N, G, NT, ST + 1, SUB>(ex, tid, kind, cb, stg, tb);
    }
  }
}

// Single-stage plans (N = R1) end in the first stage: its output goes through
// the padded tile so that the write above stays uniform.
template <typename T, int N, int G, int NT, int SUB = 1, class Exec>
QHD void ztile_after_first(Exec& ex, int tid, int kind, Cx<T>* cb, T* stg, Tables<T> tb) {
  using Z = ZTile<T, N, G, NT, SUB>;
  if constexpr (Z::plan.n_stages > 1) {
    ztile_rest<T, N, G, NT, 1, SUB>(ex, tid, kind, cb, stg, tb);
  } else {
    // the first stage wrote Z (or F) in natural order: finish like a last stage
    if (is_forward(kind)) {
      typename Z::UnpackRegs ur;
      ex.phase([&](int t, typename Z::UnpackRegs& rg) { Z::unpack_read(t, cb, tb, rg); },
               [&](int t, typename Z::UnpackRegs& rg) { Z::unpack_write(t, stg, kind, rg); }, tid, ur, true, false);
    } else {
      struct One {
        T x[(G * N + NT - 1) / NT], y[(G * N + NT - 1) / NT];
      } one;
      ex.phase(
          [&](int t, One& o) {
            for (int c = 0; c < (G * N + NT - 1) / NT; ++c) {
              const int w = t + c * NT;
              if (w >= G * N) break;
              const int g = w / N, k = w - g * N;
              const Cx<T> f = cb[g * Z::LDC + Z::phi(k)];
              o.x[c] = f.x;
              o.y[c] = f.y;
            }
          },
          [&](int t, One& o) {
            for (int c = 0; c < (G * N + NT - 1) / NT; ++c) {
              const int w = t + c * NT;
              if (w >= G * N) break;
              const int g = w / N, k = w - g * N;
              Z::put_inv(stg, kind, g, k, Cx<T>{o.x[c], o.y[c]});
            }
          },
          tid, one, true, false);
    }
  }
}

// Shared-memory copy of the full root table for the later stages: FP32 only
// (it measured neutral for FP64, whose N = 512 tile would not fit twice per SM).
template <typename T> constexpr bool zpass_root_copy() { return sizeof(T) == 4; }

#ifdef __CUDACC__
// Persistent z pass: tiles of P = 2G consecutive rows (P divides ny), N <= 512
// (N = 512 moves each row as two 256-element boxes, held [2][P][256]).
// Shared memory: two dense landing buffers (TMA loads) and the padded complex
// tile, whose first P * N elements double as the dense staging rows of the
// TMA store.  One thread issues all copies; the landing buffer of tile t is
// refilled (tile t + 2 gridDim.x) as soon as the first stage has read it, and
// the staging rows are rewritten only after the previous store has read them.
// KIND >= 0: the transform kind fixed at compile time (the launch passes the
// same value in `kind`), so every kind-dependent branch and sign folds away.
template <typename T, int N, int P, int KS, int KIND = -1>
__global__ void __launch_bounds__(256, 2)
    tma_zpass_kernel(const __grid_constant__ CUtensorMap src_map, const __grid_constant__ CUtensorMap dst_map, Geom g,
                     int kind, Tables<T> tb, int ntiles, int* err, uint32_t polls, int skip, const T* mk, int rev) {
  if constexpr (KIND >= 0) kind = KIND;
  constexpr int NT = 256, G = P / 2, SUB = (N + 255) / 256, BN = N / SUB;
  using Z = ZTile<T, N, G, NT, SUB>;
  constexpr bool kRootCopy = zpass_root_copy<T>();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* raw0 = reinterpret_cast<T*>(smem_raw);
  T* raw1 = raw0 + P * N;
  Cx<T>* cb = reinterpret_cast<Cx<T>*>(raw1 + P * N);
  T* stg = reinterpret_cast<T*>(cb);
  uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(cb) + ((Z::cb_bytes() + 15) / 16) * 16);
  // per-CTA copies of the twiddles: stage 1's as [u][b], and the quarter-wave
  // table the pre-twiddle and the unpack read
  Cx<T>* tw1 = reinterpret_cast<Cx<T>*>(bar + 2);
  Cx<T>* qt = tw1 + N;
  Cx<T>* rt = qt + N;   // FP32: the root table itself, for the later stages
  const int tid = threadIdx.x;
  {
    constexpr int M = N / Z::R1;
    for (int e = tid; e < N; e += 256) {
      const int u = e / M, b = e - u * M;
      tw1[e] = tb.root[b * u];
      qt[e] = tb.quarter[e];
      if constexpr (kRootCopy) rt[e] = tb.root[e];
    }
    tb.quarter = qt;
    if constexpr (kRootCopy) tb.root = rt;
  }
  auto origin = [&](int t, int& c1, int& c2) {
    const int row = (rev ? ntiles - 1 - t : t) * P;
    c2 = row / g.ny;
    c1 = row - c2 * g.ny;
  };
  auto issue = [&](T* dst, uint64_t* b, int t) {
    int c1, c2;
    origin(t, c1, c2);
    mbar_expect_tx(b, uint32_t(P) * N * sizeof(T));
#pragma unroll
    for (int sb = 0; sb < SUB; ++sb) tma_load_3d(dst + sb * P * BN, &src_map, b, sb * BN, c1, c2);
  };
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int t0 = blockIdx.x;
  if (tid == 0) {
    if (t0 < ntiles && t0 != skip) issue(raw0, &bar[0], t0);
    if (t0 + int(gridDim.x) < ntiles && t0 + int(gridDim.x) != skip) issue(raw1, &bar[1], t0 + gridDim.x);
  }
  DevExec ex;
  int it = 0;
  for (int t = t0; t < ntiles; t += gridDim.x, ++it) {
    const int b = it & 1;
    T* raw = b ? raw1 : raw0;
    const bool arrived = mbar_wait_bounded(&bar[b], (it >> 1) & 1, polls);
    if (!__syncthreads_and(arrived)) {
      if (tid == 0) atomicExch(err, 1);
      drain_other(bar, b, it, t, int(gridDim.x), ntiles, skip, polls);
      break;
    }
    // first stage: dense rows -> registers | previous store read out | -> padded tile
    typename Z::template Regs<Z::R1> r1;
    Z::first_read(tid, typename Z::template RowsK<KS>{raw, mk}, kind, tb, r1, tw1);
    if (tid == 0) bulk_wait_read0();
    __syncthreads();
    if (tid == 0 && t + 2 * int(gridDim.x) < ntiles && t + 2 * int(gridDim.x) != skip) {
      fence_proxy_async_smem();
      issue(raw, &bar[b], t + 2 * gridDim.x);
    }
    Z::template stage_write<Z::R1, 1>(tid, cb, r1);
    __syncthreads();
    ztile_after_first<T, N, G, NT, SUB>(ex, tid, kind, cb, stg, tb);
    // this thread's staging writes to the async proxy, then every thread's
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      int c1, c2;
      origin(t, c1, c2);
#pragma unroll
      for (int sb = 0; sb < SUB; ++sb) tma_store_3d(&dst_map, stg + sb * P * BN, sb * BN, c1, c2);
      bulk_commit();
    }
  }
  if (tid == 0) bulk_wait0();
}

// ---------------------------------------------------------------------------
// Warp-tile z pass: every warp is an independent pipeline over its own tiles
// of 2G rows (G complex pencils: 2 in float, 1 in double).  It loads its rows
// with its own TMA copies (two landing buffers, two mbarriers), runs the tile
// FFT of ZTile with warp-wide synchronisation only (its padded complex tile
// is its own), stages the output rows over that tile and stores them with
// its own TMA store.  No CTA barrier after the set-up: warps never wait for
// each other, so one warp's FFT overlaps the others' copies.
// ---------------------------------------------------------------------------
template <typename T> constexpr int zw_pencils() { return sizeof(T) == 4 ? 2 : 1; }
constexpr int kZwWarps = 8;

template <typename T, int N>
struct ZwLayout {
  static constexpr int G = zw_pencils<T>(), R = 2 * G;          // pencils, rows per warp tile
  using Z = ZTile<T, N, G, 32, 1>;
  static constexpr int RAW = R * N;                              // elements of one landing buffer
  static constexpr int WB = int(((Z::cb_bytes() + 127) / 128) * 128);   // work bytes per warp
  static constexpr size_t raw_bytes() { return size_t(kZwWarps) * 2 * RAW * sizeof(T); }
  static constexpr size_t smem_bytes() {
    return raw_bytes() + size_t(kZwWarps) * WB + 2 * kZwWarps * 8 + (zpass_root_copy<T>() ? 3 : 2) * N * sizeof(Cx<T>);
  }
  static_assert(size_t(R) * N * sizeof(T) <= size_t(WB), "the staging rows overlay the warp's tile");
};

template <typename T, int N, int KS, int KIND = -1>
__global__ void __launch_bounds__(256, 2)
    tma_zpass_warp_kernel(const __grid_constant__ CUtensorMap src_map, const __grid_constant__ CUtensorMap dst_map,
                          Geom g, int kind, Tables<T> tb, int ntiles, int* err, uint32_t polls, int skip,
                          const T* mk, int rev) {
  if constexpr (KIND >= 0) kind = KIND;
  using L = ZwLayout<T, N>;
  using Z = typename L::Z;
  constexpr int G = L::G, R = L::R, RAW = L::RAW;
  constexpr bool kRootCopy = zpass_root_copy<T>();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  T* raw = reinterpret_cast<T*>(smem_raw) + size_t(warp) * 2 * RAW;   // this warp's landing buffers
  unsigned char* work_base = smem_raw + L::raw_bytes();
  Cx<T>* cb = reinterpret_cast<Cx<T>*>(work_base + size_t(warp) * L::WB);
  T* stg = reinterpret_cast<T*>(cb);
  uint64_t* bars = reinterpret_cast<uint64_t*>(work_base + size_t(kZwWarps) * L::WB);
  uint64_t* bar = bars + 2 * warp;
  Cx<T>* tw1 = reinterpret_cast<Cx<T>*>(bars + 2 * kZwWarps);
  Cx<T>* qt = tw1 + N;
  Cx<T>* rt = qt + N;
  {
    constexpr int M = N / Z::R1;
    for (int e = tid; e < N; e += 256) {
      const int u = e / M, b = e - u * M;
      tw1[e] = tb.root[b * u];
      qt[e] = tb.quarter[e];
      if constexpr (kRootCopy) rt[e] = tb.root[e];
    }
    tb.quarter = qt;
    if constexpr (kRootCopy) tb.root = rt;
  }
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();   // tables and barriers ready: the only CTA-wide barrier
  const int w0 = int(blockIdx.x) * kZwWarps + warp, nwarps = int(gridDim.x) * kZwWarps;
  auto origin = [&](int t, int& c1, int& c2) {
    const int row = (rev ? ntiles - 1 - t : t) * R;   // R rows of one x plane (R divides ny)
    c2 = row / g.ny;
    c1 = row - c2 * g.ny;
  };
  auto issue = [&](int b, int t) {
    int c1, c2;
    origin(t, c1, c2);
    mbar_expect_tx(&bar[b], uint32_t(RAW * sizeof(T)));
    tma_load_3d(raw + b * RAW, &src_map, &bar[b], 0, c1, c2);
  };
  if (lane == 0) {
    if (w0 < ntiles && w0 != skip) issue(0, w0);
    if (w0 + nwarps < ntiles && w0 + nwarps != skip) issue(1, w0 + nwarps);
  }
  WarpExec ex;
  int it = 0;
  for (int t = w0; t < ntiles; t += nwarps, ++it) {
    const int b = it & 1;
    const bool arrived = mbar_wait_bounded(&bar[b], (it >> 1) & 1, polls);
    if (!__all_sync(0xffffffffu, arrived)) {
      if (lane == 0) atomicExch(err, 1);
      const int t_other = t + nwarps;   // drain the other buffer's copy
      if (t_other < ntiles && t_other != skip) mbar_wait_bounded(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
      break;
    }
    typename Z::template Regs<Z::R1> r1;
    Z::first_read(lane, typename Z::template RowsK<KS>{raw + b * RAW, mk}, kind, tb, r1, tw1);
    if (lane == 0) bulk_wait_read0();   // the previous store has read the staging rows
    __syncwarp();
    const int tn = t + 2 * nwarps;
    if (lane == 0 && tn < ntiles && tn != skip) {
      fence_proxy_async_smem();
      issue(b, tn);
    }
    Z::template stage_write<Z::R1, 1>(lane, cb, r1);
    __syncwarp();
    ztile_after_first<T, N, G, 32, 1>(ex, lane, kind, cb, stg, tb);
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      int c1, c2;
      origin(t, c1, c2);
      tma_store_3d(&dst_map, stg, 0, c1, c2);
      bulk_commit();
    }
  }
  if (lane == 0) bulk_wait0();
}

template <typename T, int N, int KS>
cudaError_t launch_zpass_warp(const Geom& g, int kind, Tables<T> tb, const T* src, T* dst, cudaStream_t s,
                              const T* mk) {
  using L = ZwLayout<T, N>;
  if (g.ny % L::R != 0) return cudaErrorNotSupported;
  const uint32_t box[3] = {uint32_t(N), uint32_t(L::R), 1};
  CUtensorMap smap, dmap;
  if (!MapCache::get().lookup(&smap, src, int(sizeof(T)), g.nx, g.ny, g.nz, 2, box) ||
      !MapCache::get().lookup(&dmap, dst, int(sizeof(T)), g.nx, g.ny, g.nz, 2, box))
    return cudaErrorNotSupported;
  const size_t smem = L::smem_bytes();
  // the kind fixed at compile time (kFixedKind lengths)
  using K = decltype(&tma_zpass_warp_kernel<T, N, KS>);
  K kern = &tma_zpass_warp_kernel<T, N, KS>;
  if constexpr (kFixedKind<N>) {
    const K ks[4] = {&tma_zpass_warp_kernel<T, N, KS, E10>, &tma_zpass_warp_kernel<T, N, KS, E01>,
                     &tma_zpass_warp_kernel<T, N, KS, O10>, &tma_zpass_warp_kernel<T, N, KS, O01>};
    kern = ks[kind & 3];
  }
  static int per_sm_k[5] = {};   // per instantiation: the runtime-kind kernel, then one per fixed kind
  int& per_sm = per_sm_k[kFixedKind<N> ? 1 + (kind & 3) : 0];
  if (per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 256, smem);
    if (e != cudaSuccess) return e;
    per_sm = n > 0 ? n : 1;
  }
  const int tiles = (g.nx * g.ny) / L::R;
  const int warps = per_sm * tma_config().sms * kZwWarps;
  const int grid = tiles < warps ? (tiles + kZwWarps - 1) / kZwWarps : per_sm * tma_config().sms;
  kern<<<grid, 256, smem, s>>>(smap, dmap, g, kind, tb, tiles, tma_config().err, tma_config().poll_limit,
                               tma_config().skip_tile, mk, int(tma_config().zrev));
  return cudaGetLastError();
}

#ifndef QUASI_ZPASS
#define QUASI_ZPASS 1
#endif

template <typename T, int N, int KS>
cudaError_t launch_zpass_nk(const Geom& g, int kind, Tables<T> tb, const T* src, T* dst, cudaStream_t s,
                            const T* mk) {
  constexpr int P = pass_pencils<T>(N), G = P / 2, SUB = (N + 255) / 256;
  using Z = ZTile<T, N, G, 256, SUB>;
  if (g.ny % P != 0) return cudaErrorNotSupported;
  const uint32_t box[3] = {uint32_t(N / SUB), uint32_t(P), 1};
  CUtensorMap smap, dmap;
  if (!MapCache::get().lookup(&smap, src, int(sizeof(T)), g.nx, g.ny, g.nz, 2, box) ||
      !MapCache::get().lookup(&dmap, dst, int(sizeof(T)), g.nx, g.ny, g.nz, 2, box))
    return cudaErrorNotSupported;
  const size_t smem = size_t(2) * P * N * sizeof(T) + ((Z::cb_bytes() + 15) / 16) * 16 + 16 +
                      (zpass_root_copy<T>() ? 3 : 2) * N * sizeof(Cx<T>);
  using K = decltype(&tma_zpass_kernel<T, N, P, KS>);
  K kern = &tma_zpass_kernel<T, N, P, KS>;
  if constexpr (kFixedKind<N>) {
    const K ks[4] = {&tma_zpass_kernel<T, N, P, KS, E10>, &tma_zpass_kernel<T, N, P, KS, E01>,
                     &tma_zpass_kernel<T, N, P, KS, O10>, &tma_zpass_kernel<T, N, P, KS, O01>};
    kern = ks[kind & 3];
  }
  static int per_sm_k[5] = {};   // per instantiation: the runtime-kind kernel, then one per fixed kind
  int& per_sm = per_sm_k[kFixedKind<N> ? 1 + (kind & 3) : 0];
  if (per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 256, smem);
    if (e != cudaSuccess) return e;
    per_sm = n > 0 ? n : 1;
  }
  const int tiles = (g.nx * g.ny) / P;
  const int grid = tiles < per_sm * tma_config().sms ? tiles : per_sm * tma_config().sms;
  kern<<<grid, 256, smem, s>>>(smap, dmap, g, kind, tb, tiles, tma_config().err, tma_config().poll_limit,
                               tma_config().skip_tile, mk, int(tma_config().zrev));
  return cudaGetLastError();
}

// ks: 0 plain, 1 row[k + 1], 2 row[k + 1] times -mk[k] (double passes only)
template <typename T, int N>
cudaError_t launch_zpass_n(const Geom& g, int kind, Tables<T> tb, const T* src, T* dst, cudaStream_t s, int ks,
                           const T* mk) {
  if (ks == 2 && (sizeof(T) != 8 || !mk)) return cudaErrorNotSupported;
  if constexpr (N >= 64 && N <= 256) {
    if (tma_config().zwarp[sizeof(T) == 8]) {
      cudaError_t e;
      if (ks == 0) e = launch_zpass_warp<T, N, 0>(g, kind, tb, src, dst, s, mk);
      else if (ks == 1) e = launch_zpass_warp<T, N, 1>(g, kind, tb, src, dst, s, mk);
      else if constexpr (sizeof(T) == 8) e = launch_zpass_warp<T, N, 2>(g, kind, tb, src, dst, s, mk);
      else e = cudaErrorNotSupported;
      if (e != cudaErrorNotSupported) return e;
    }
  }
  if (ks == 0) return launch_zpass_nk<T, N, 0>(g, kind, tb, src, dst, s, mk);
  if (ks == 1) return launch_zpass_nk<T, N, 1>(g, kind, tb, src, dst, s, mk);
  if constexpr (sizeof(T) == 8) return launch_zpass_nk<T, N, 2>(g, kind, tb, src, dst, s, mk);
  return cudaErrorNotSupported;
}

// z pass src -> dst (plain fields; ks = 1 transforms row[k + 1], zero at the
// top; ks = 2 also multiplies it by -mk[k]) on the TMA load/store kernel;
// cudaErrorNotSupported when the shape or configuration does not allow it
// (the caller takes the general pass).
template <typename T>
cudaError_t launch_zpass(const Geom& g, int kind, Tables<T> tb, const T* src, T* dst, cudaStream_t s, int ks = 0,
                         const T* mk = nullptr) {
  if (!QUASI_ZPASS || !tma_config().enabled || !tma_config().err) return cudaErrorNotSupported;
  switch (g.nz) {
    case 16: return launch_zpass_n<T, 16>(g, kind, tb, src, dst, s, ks, mk);
    case 32: return launch_zpass_n<T, 32>(g, kind, tb, src, dst, s, ks, mk);
    case 64: return launch_zpass_n<T, 64>(g, kind, tb, src, dst, s, ks, mk);
    case 96: return launch_zpass_n<T, 96>(g, kind, tb, src, dst, s, ks, mk);
    case 128: return launch_zpass_n<T, 128>(g, kind, tb, src, dst, s, ks, mk);
    case 192: return launch_zpass_n<T, 192>(g, kind, tb, src, dst, s, ks, mk);
    case 256: return launch_zpass_n<T, 256>(g, kind, tb, src, dst, s, ks, mk);
    case 512: return launch_zpass_n<T, 512>(g, kind, tb, src, dst, s, ks, mk);
    default: return cudaErrorNotSupported;
  }
}
#endif

}  // namespace quasi
