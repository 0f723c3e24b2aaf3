// One axis pass of a 3-D r2r transform: every CTA stages a tile of P pencils
// along one axis in shared memory, transforms them (r2r_core.cuh) and writes
// them back.  A 3-D transform is three such passes; pointwise work is fused
// into the first pass's loader and the last pass's storer, so intermediate
// real or spectral fields that the reference materialises (quasi.cpp keeps
// 39 arrays and copies each through `trans_local`) are computed on the fly.
//
// Tile geometry on the reference layout a[(i*Ny + j)*Nz + k] (z contiguous):
//   AXIS 2 (z): P consecutive rows (i, j), pencil = row, n = k      (coalesced)
//   AXIS 1 (y): fixed i, P consecutive k; pencil = column k, n = j
//   AXIS 0 (x): fixed j, P consecutive k; pencil = column k, n = i
// Loader:  T operator()(int i, int j, int k) const   value entering the pass
// Storer:  void operator()(int i, int j, int k, T v) const   value leaving it
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "r2r_core.cuh"
#include "tc_pass.cuh"
#include "tma.cuh"

namespace quasi {

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

struct DevExec {
  template <class R, class W, class Regs>
  __device__ __forceinline__ void phase(R&& rd, W&& wr, int tid, Regs& regs, bool mid, bool after) {
    rd(tid, regs);
    if (mid) __syncthreads();
    wr(tid, regs);
    if (after) __syncthreads();
  }
  __device__ __forceinline__ void sync() { __syncthreads(); }
};

// The same phases synchronised within one warp only (warp-tile kernels, whose
// tiles belong to one warp).
struct WarpExec {
  template <class R, class W, class Regs>
  __device__ __forceinline__ void phase(R&& rd, W&& wr, int tid, Regs& regs, bool mid, bool after) {
    rd(tid, regs);
    if (mid) __syncwarp();
    wr(tid, regs);
    if (after) __syncwarp();
  }
  __device__ __forceinline__ void sync() { __syncwarp(); }
};

struct Geom {
  int nx, ny, nz;
};

// ---------------------------------------------------------------------------
// Plain loaders / storers
// ---------------------------------------------------------------------------
__device__ __forceinline__ size_t lin(const Geom& g, int i, int j, int k) {
  return (size_t(i) * g.ny + j) * g.nz + k;
}

template <typename T>
struct LoadField {
  Geom g;
  const T* src;
  __device__ T operator()(int i, int j, int k) const { return src[lin(g, i, j, k)]; }
  // k even: one aligned vector load of (k, k+1)
  __device__ void pair(int i, int j, int k, T& a, T& b) const {
    const auto v = *reinterpret_cast<const typename Vec2<T>::type*>(src + lin(g, i, j, k));
    a = v.x;
    b = v.y;
  }
};

template <typename T>
struct StoreField {
  Geom g;
  T* dst;
  __device__ void operator()(int i, int j, int k, T v) const { dst[lin(g, i, j, k)] = v; }
  __device__ void pair(int i, int j, int k, T a, T b) const {
    typename Vec2<T>::type v;
    v.x = a;
    v.y = b;
    *reinterpret_cast<typename Vec2<T>::type*>(dst + lin(g, i, j, k)) = v;
  }
};

template <class S> struct IsStoreField : std::false_type {};
template <typename T> struct IsStoreField<StoreField<T>> : std::true_type {};

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double2; };

template <typename T>
struct ScaleStore {
  Geom g;
  T* dst;
  T s;
  __device__ T value(int, int, int, T v) const { return v * s; }
  __host__ __device__ T* stage_dst() const { return dst; }
  __device__ void operator()(int i, int j, int k, T v) const { dst[lin(g, i, j, k)] = value(i, j, k, v); }
};

// Storers that map a value before it lands (value(i, j, k, v)) in one field
// (stage_dst()): their x / y tiles can be staged and TMA-stored as well.
template <class S, class = void> struct HasStageValue : std::false_type {};
template <class S> struct HasStageValue<S, std::void_t<decltype(&S::stage_dst)>> : std::true_type {};


template <int AXIS>
__device__ __forceinline__ void tile_coords(const Geom& g, int tile, int P, int p, int n, int& i, int& j, int& k) {
  if (AXIS == 2) {
    const int row = tile * P + p;
    i = row / g.ny;
    j = row - i * g.ny;
    k = n;
  } else {
    const int kt = g.nz / P;
    const int outer = tile / kt;
    k = (tile - outer * kt) * P + p;
    if (AXIS == 1) { i = outer; j = n; }
    else { j = outer; i = n; }
  }
}

// Element e of a z tile -> (pencil p, position n), n fastest (contiguous rows).
template <int P, int N>
__device__ __forceinline__ void z_elem(int e, int& p, int& n) {
  p = e / N;
  n = e - p * N;
}

// Paired access to k and k+1 (k even): the two real pencils of one complex
// pencil in an x or y tile.  Loaders/storers may provide pair() themselves
// (vector access); otherwise the element operator is called twice.
template <class L, class = void> struct HasPair : std::false_type {};
template <class L> struct HasPair<L, std::void_t<decltype(&L::pair)>> : std::true_type {};

template <typename T, class Load>
__device__ __forceinline__ void load_pair(const Load& ld, int i, int j, int k, T& a, T& b) {
  if constexpr (HasPair<Load>::value) ld.pair(i, j, k, a, b);
  else { a = ld(i, j, k); b = ld(i, j, k + 1); }
}

template <typename T, class Store>
__device__ __forceinline__ void store_pair(const Store& st, int i, int j, int k, T a, T b) {
  if constexpr (HasPair<Store>::value) st.pair(i, j, k, a, b);
  else { st(i, j, k, a); st(i, j, k + 1, b); }
}

// x/y tiles read and write global memory directly from the FFT stages
template <typename T, int AXIS, class Load>
struct GlobSrc {
  Load ld;
  int outer, k0;
  __device__ __forceinline__ void pair(int g, int n, T& a, T& b) const {
    const int k = k0 + 2 * g;
    if (AXIS == 1) load_pair<T>(ld, outer, n, k, a, b);
    else load_pair<T>(ld, n, outer, k, a, b);
  }
};

template <typename T, int AXIS, class Store>
struct GlobSnk {
  Store st;
  int outer, k0;
  __device__ __forceinline__ void put(int g, int n, T a, T b) const {
    const int k = k0 + 2 * g;
    if constexpr (IsStoreField<Store>::value) {
      // plain field: (outer, n) -> element offset without 64-bit index math per pair
      const Geom& gm = st.g;
      const size_t row = AXIS == 1 ? size_t(outer) * gm.ny + n : size_t(n) * gm.ny + outer;
      typename Vec2<T>::type v;
      v.x = a;
      v.y = b;
      *reinterpret_cast<typename Vec2<T>::type*>(st.dst + row * gm.nz + k) = v;
    } else if (AXIS == 1) {
      store_pair<T>(st, outer, n, k, a, b);
    } else {
      store_pair<T>(st, n, outer, k, a, b);
    }
  }
};

// Threads per CTA and the CTAs per SM the register allocation must allow.
template <typename T> constexpr int pass_threads() { return 256; }
template <typename T> constexpr int pass_min_blocks() { return 2; }

template <typename T, int N, int AXIS, int P, class Load, class Store>
__global__ void __launch_bounds__(pass_threads<T>(), pass_min_blocks<T>()) axis_pass_kernel(Geom g, int kind, Tables<T> tb, Load ld,
                                                                      Store st) {
  constexpr int NT = pass_threads<T>();
  constexpr int LD = tile_ld(N);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* buf = reinterpret_cast<T*>(smem_raw);
  const int tile = blockIdx.x;
  const int tid = threadIdx.x;
  DevExec ex;
  if constexpr (AXIS != 2) {
    // x / y: P consecutive k columns; first stage loads from global, an inverse
    // kind's last stage (or a forward kind's unpack) stores to global
    const int kt = g.nz / P;
    const int outer = tile / kt, k0 = (tile - outer * kt) * P;
    r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(buf),
                                      GlobSrc<T, AXIS, Load>{ld, outer, k0}, GlobSnk<T, AXIS, Store>{st, outer, k0}, tb);
  } else {
    // z: P contiguous rows staged through shared memory (coalesced both ways)
    constexpr int E = P * N;
    constexpr int PER = (E + NT - 1) / NT;
    constexpr int B = PER < 16 ? PER : 16;
#pragma unroll
    for (int c0 = 0; c0 < PER; c0 += B) {
      T v[B];
#pragma unroll
      for (int c = 0; c < B; ++c) {
        const int e = tid + (c0 + c) * NT;
        if ((E % NT == 0 && PER % B == 0) || (c0 + c < PER && e < E)) {
          int p, n, i, j, k;
          z_elem<P, N>(e, p, n);
          tile_coords<2>(g, tile, P, p, n, i, j, k);
          v[c] = ld(i, j, k);
        }
      }
#pragma unroll
      for (int c = 0; c < B; ++c) {
        const int e = tid + (c0 + c) * NT;
        if ((E % NT == 0 && PER % B == 0) || (c0 + c < PER && e < E)) {
          int p, n;
          z_elem<P, N>(e, p, n);
          buf[p * LD + n] = v[c];
        }
      }
    }
    __syncthreads();
    r2r_tile_inplace<T, N, P / 2, NT>(ex, tid, kind, buf, tb);
#pragma unroll
    for (int c = 0; c < PER; ++c) {
      const int e = tid + c * NT;
      if (E % NT == 0 || e < E) {
        int p, n, i, j, k;
        z_elem<P, N>(e, p, n);
        tile_coords<2>(g, tile, P, p, n, i, j, k);
        st(i, j, k, buf[p * LD + n]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Persistent TMA-pipelined pass for plain field loads.
//
// Each CTA walks tiles t = blockIdx.x, + gridDim.x, ...  Two raw buffers
// receive whole tiles by cp.async.bulk.tensor (one thread issues, an mbarrier
// counts the bytes); the copy of tile t + 2*gridDim.x is issued as soon as
// tile t's raw buffer has been consumed, so the memory system always has the
// next tile in flight while the current one is transformed.
//   x / y: the box (P k, N rows) lands as raw[n * P + p]; adjacent k pencils
//          2g, 2g+1 are one complex value, read directly by the first stage.
//   z:     the box (N k, P rows) lands as raw[p * N + n] and is copied into
//          the padded in-place tile.
// A wait that does not complete within its poll limit sets *err and leaves
// the tile loop (the host reports the error after the step).
// ---------------------------------------------------------------------------
template <typename T>
struct RawSrc {
  const T* raw;
  int P;
  QHD void pair(int g, int n, T& a, T& b) const {
    const typename Vec2<T>::type v = *reinterpret_cast<const typename Vec2<T>::type*>(raw + n * P + 2 * g);
    a = v.x;
    b = v.y;
  }
};

// x / y tile sink for a TMA store: pencils 2g, 2g+1 at position n into the
// staging rows [n][P] (the store box's layout), which overlay the work tile.
template <typename T>
struct RowStageSnk {
  static constexpr bool kAliasesTile = true;
  T* stg;
  int P;
  QHD void put(int g, int n, T a, T b) const {
    typename Vec2<T>::type v;
    v.x = a;
    v.y = b;
    *reinterpret_cast<typename Vec2<T>::type*>(stg + n * P + 2 * g) = v;
  }
};

// The same for a storer with value(i, j, k, v): the mapped values are staged.
template <typename T, int AXIS, class Store>
struct RowStageValSnk {
  static constexpr bool kAliasesTile = true;
  T* stg;
  int P, outer, k0;
  Store st;
  __device__ void put(int g, int n, T a, T b) const {
    const int k = k0 + 2 * g;
    const int i = AXIS == 1 ? outer : n, j = AXIS == 1 ? n : outer;
    typename Vec2<T>::type v;
    v.x = st.value(i, j, k, a);
    v.y = st.value(i, j, k + 1, b);
    *reinterpret_cast<typename Vec2<T>::type*>(stg + n * P + 2 * g) = v;
  }
};

// Identity multiplier (plain passes).
struct NoMul {
  static constexpr bool kActive = false;
  template <int AX> static constexpr bool kTable = false;
  __device__ double operator()(int, int, int) const { return 1.0; }
};

// Axis tables.  A multiplier whose dependence on the index n along a pass's
// axis AX goes through one double wavenumber table sets kTable<AX> and gives
//   const double* axis_table(int ax)         the table (N entries)
//   Col col_at(int ax, int outer, int k)      the rest, once per pencil
//   double from(int ax, double w, const Col&)  the multiplier, w = table[n]
// The x / y kernels copy the table into shared memory once per CTA (when two
// CTAs per SM still fit), so the per-element work reads shared memory only.
template <class M, int AX> constexpr bool axis_tab() { return M::kActive && M::template kTable<AX>; }

// Tables a pass kernel stages: one per multiplier, 0 unless every active
// multiplier has one on this axis and the kernel still fits twice per SM.
template <int AX, class Mul, class Mul2>
constexpr int row_tables(size_t base_smem, int n) {
  constexpr bool dual = Mul2::kActive;
  constexpr int want = axis_tab<Mul, AX>() && (!dual || axis_tab<Mul2, AX>()) ? (dual ? 2 : 1) : 0;
  return want && 2 * (base_smem + size_t(want) * n * sizeof(double) + 1024) <= 233472 ? want : 0;
}

template <class M, class = void> struct MulCol { struct type {}; };
template <class M> struct MulCol<M, std::void_t<typename M::Col>> { using type = typename M::Col; };

// x / y tile source with a per-element multiplier of the OUTPUT index
// (i, j, k): the spectral prologue of an inverse transform.
template <typename T, int AXIS, class Mul, bool ALIAS = false, bool TAB = false>
struct MulSrc {
  static constexpr bool kAliasesTile = ALIAS;
  const T* raw;
  int P, outer, k0;
  Mul mul;
  // x passes (and TAB): the column parts of this thread's two pencils (prep)
  typename MulCol<Mul>::type ca{}, cb{};
  const double* tab = nullptr;   // TAB: the multiplier's axis table in shared memory
  // gt = the one pencil pair this thread reads: the first stage's pencil-fastest
  // mapping gives g = tid % (P/2) whenever the thread count is a multiple of P/2
  __device__ void prep(int gt) {
    if constexpr (TAB) {
      ca = mul.col_at(AXIS, outer, k0 + 2 * gt);
      cb = mul.col_at(AXIS, outer, k0 + 2 * gt + 1);
    } else if constexpr (Mul::kActive && AXIS == 0) {
      ca = mul.col(outer, k0 + 2 * gt);
      cb = mul.col(outer, k0 + 2 * gt + 1);
    }
  }
  QHD void pair(int g, int n, T& a, T& b) const {
    const typename Vec2<T>::type v = *reinterpret_cast<const typename Vec2<T>::type*>(raw + n * P + 2 * g);
    a = v.x;
    b = v.y;
    if constexpr (Mul::kActive) {
      // the multiplier is evaluated in its own type (double where q0^2 - q^2
      // cancels), rounded to the storage type once, and applied there
      if constexpr (TAB) {
        const double w = tab[n];
        a *= T(mul.from(AXIS, w, ca));
        b *= T(mul.from(AXIS, w, cb));
      } else if constexpr (AXIS == 0) {
        a *= T(mul.row(n, ca));
        b *= T(mul.row(n, cb));
      } else {
        const int k = k0 + 2 * g;
        a *= T(mul(outer, n, k));
        b *= T(mul(outer, n, k + 1));
      }
    }
  }
};

constexpr uint32_t kTmaPollLimit = 1u << 24;

// After a timed-out wait on buffer b for tile t: the other buffer holds the
// copy of tile t + stride unless that tile is past the end or was skipped by
// the fault-injection hook; wait for it (bounded) so that no copy into this
// CTA's shared memory is in flight when the CTA exits.
__device__ __forceinline__ void drain_other(uint64_t* bar, int b, int it, int t, int stride, int ntiles, int skip,
                                            uint32_t polls) {
  const int t_other = t + stride;
  if (t_other < ntiles && t_other != skip) mbar_wait_bounded(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
}

template <int AXIS, int P>
__device__ __forceinline__ void tile_origin(const Geom& g, int tile, int& c0, int& c1, int& c2) {
  if (AXIS == 2) {   // P rows (i, j0..j0+P-1); P divides ny
    const int row = tile * P;
    c2 = row / g.ny;
    c1 = row - c2 * g.ny;
    c0 = 0;
  } else {
    const int kt = g.nz / P;
    const int outer = tile / kt;
    c0 = (tile - outer * kt) * P;
    if (AXIS == 1) { c2 = outer; c1 = 0; }
    else { c1 = outer; c2 = 0; }
  }
}

template <typename T, int N, int AXIS, int P>
__device__ __forceinline__ void tma_issue_tile(const CUtensorMap* map, T* raw, uint64_t* bar, const Geom& g, int tile,
                                               int dc1, int dc2) {
  constexpr int SUB = (N + 255) / 256;     // boxes per tile along the transform axis (box dims <= 256)
  constexpr int BN = N / SUB;
  int c0, c1, c2;
  tile_origin<AXIS, P>(g, tile, c0, c1, c2);
  c1 += dc1;   // shifted loads (j + 1, i + 1): out-of-range rows read as zero
  c2 += dc2;
  mbar_expect_tx(bar, uint32_t(P) * N * sizeof(T));
#pragma unroll
  for (int sb = 0; sb < SUB; ++sb) {
    if (AXIS == 2) tma_load_3d(raw + sb * BN, map, bar, c0 + sb * BN, c1, c2);          // only N <= 256 reaches here
    else if (AXIS == 1) tma_load_3d(raw + sb * BN * P, map, bar, c0, c1 + sb * BN, c2);
    else tma_load_3d(raw + sb * BN * P, map, bar, c0, c1, c2 + sb * BN);
  }
}

template <typename T> constexpr int tma_threads() { return 256; }
// Transform lengths whose TMA pass kernels take the kind as a template
// parameter (one instantiation per kind; shorter ones take it at run time).
template <int N> constexpr bool kFixedKind = N >= 64;

template <typename T, int N, int P> constexpr int tma_work_elems() { return ((P * tile_ld(N) + 15) / 16) * 16; }

// Mul2 != NoMul (x / y): each tile, loaded once, is transformed twice,
// with mul into st and with mul2 into st2 (two inverse transforms of the same
// spectral field that differ only in their multiplier).
// TSTORE (plain field outputs): the last stage writes the staging rows
// over the work tile and one thread stores the tile through dmap (dmap2 for
// the dual pass's second output); the next tile's first stage waits for the
// store to have read them.
// KIND >= 0: the transform kind fixed at compile time (the launch passes the
// same value in `kind`), so every kind-dependent branch and sign folds away.
template <typename T, int N, int AXIS, int P, class Store, class Mul, class Mul2 = NoMul, bool TSTORE = false,
          int TABS = 0, int KIND = -1>
__global__ void __launch_bounds__(tma_threads<T>(), 2)
    tma_pass_kernel(const __grid_constant__ CUtensorMap map, Geom g, int kind, Tables<T> tb, Store st, int ntiles,
                    int* err, uint32_t polls, int skip, Mul mul, int dc1, int dc2, int ks, Store st2, Mul2 mul2,
                    const __grid_constant__ CUtensorMap dmap, const __grid_constant__ CUtensorMap dmap2) {
  if constexpr (KIND >= 0) kind = KIND;
  static_assert(!TSTORE || AXIS != 2, "TMA-stored tiles are x / y passes");
  constexpr bool kDual = !std::is_same<Mul2, NoMul>::value;
  static_assert(!TSTORE || !kDual || IsStoreField<Store>::value, "dual passes stage plain fields");
  static_assert(tma_threads<T>() % (P / 2) == 0, "MulSrc::prep: each thread reads one pencil pair");
  static_assert(!kDual || AXIS != 2, "dual tiles are x / y passes");
  constexpr int NT = tma_threads<T>();
  constexpr int LD = tile_ld(N);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* raw0 = reinterpret_cast<T*>(smem_raw);
  T* raw1 = raw0 + P * N;
  T* work = raw1 + P * N;
  uint64_t* bar = reinterpret_cast<uint64_t*>(work + tma_work_elems<T, N, P>());
  double* atab = reinterpret_cast<double*>(reinterpret_cast<Cx<T>*>(bar + 2) + 2 * N);
  const int tid = threadIdx.x;
  {
    // per-CTA shared-memory copies of the twiddle tables (N entries each)
    // and of the multipliers' axis tables (TABS of N doubles)
    Cx<T>* rt = reinterpret_cast<Cx<T>*>(bar + 2);
    Cx<T>* qt = rt + N;
    for (int e = tid; e < N; e += NT) {
      rt[e] = tb.root[e];
      qt[e] = tb.quarter[e];
      if constexpr (TABS > 0) atab[e] = mul.axis_table(AXIS)[e];
      if constexpr (TABS > 1) atab[N + e] = mul2.axis_table(AXIS)[e];
    }
    tb.root = rt;
    tb.quarter = qt;
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int t0 = blockIdx.x;
  if (tid == 0) {
    // skip: the tile whose copy the fault-injection hook never issues (its
    // wait then runs out); -1 outside the failure-detection tests
    if (t0 < ntiles && t0 != skip) tma_issue_tile<T, N, AXIS, P>(&map, raw0, &bar[0], g, t0, dc1, dc2);
    if (t0 + int(gridDim.x) < ntiles)
      if (t0 + int(gridDim.x) != skip) tma_issue_tile<T, N, AXIS, P>(&map, raw1, &bar[1], g, t0 + gridDim.x, dc1, dc2);
  }
  DevExec ex;
  int it = 0;
  for (int t = t0; t < ntiles; t += gridDim.x, ++it) {
    const int b = it & 1;
    T* raw = b ? raw1 : raw0;
    const uint32_t parity = (it >> 1) & 1;
    // every thread polls; the CTA leaves together if any poll gave up
    const bool arrived = mbar_wait_bounded(&bar[b], parity, polls);
    if constexpr (TSTORE) {
      if (tid == 0) bulk_wait_read0();   // the previous tile's store has read the work tile
    }
    if (!__syncthreads_and(arrived)) {
      if (tid == 0) atomicExch(err, 1);
      drain_other(bar, b, it, t, int(gridDim.x), ntiles, skip, polls);
      break;
    }
    const int t_next = t + 2 * int(gridDim.x);
    // TSTORE: hand the staging rows over the work tile to the async proxy and
    // store them as the tile's box(es)
    auto store_tile = [&](const CUtensorMap* dm) {
      fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0) {
        constexpr int SUB = (N + 255) / 256, BN = N / SUB;
        int c0, c1, c2;
        tile_origin<AXIS, P>(g, t, c0, c1, c2);
#pragma unroll
        for (int sb = 0; sb < SUB; ++sb) {
          if (AXIS == 1) tma_store_3d(dm, work + sb * BN * P, c0, c1 + sb * BN, c2);
          else tma_store_3d(dm, work + sb * BN * P, c0, c1, c2 + sb * BN);
        }
        bulk_commit();
      }
    };
    auto issue_next = [&]() {
      if (tid == 0 && t_next < ntiles && t_next != skip) {
        fence_proxy_async_smem();
        tma_issue_tile<T, N, AXIS, P>(&map, raw, &bar[b], g, t_next, dc1, dc2);
      }
    };
    if constexpr (AXIS != 2 && kDual) {
      const int kt = g.nz / P;
      const int outer = t / kt, k0 = (t - outer * kt) * P;
      MulSrc<T, AXIS, Mul, false, (TABS > 0)> src{raw, P, outer, k0, mul};
      src.tab = atab;
      src.prep(tid % (P / 2));
      if constexpr (TSTORE) {
        r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(work), src,
                                          RowStageSnk<T>{work, P}, tb);
        store_tile(&dmap);
        if (tid == 0) bulk_wait_read0();
      } else {
        r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(work), src,
                                          GlobSnk<T, AXIS, Store>{st, outer, k0}, tb);
      }
      __syncthreads();   // the second transform rewrites the work tile
      MulSrc<T, AXIS, Mul2, false, (TABS > 1)> src2{raw, P, outer, k0, mul2};
      src2.tab = atab + N;
      src2.prep(tid % (P / 2));
      if constexpr (TSTORE) {
        r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(work), src2,
                                          RowStageSnk<T>{work, P}, tb, issue_next);
        store_tile(&dmap2);
      } else {
        r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(work), src2,
                                          GlobSnk<T, AXIS, Store>{st2, outer, k0}, tb, issue_next);
      }
    } else if constexpr (AXIS != 2) {
      const int kt = g.nz / P;
      const int outer = t / kt, k0 = (t - outer * kt) * P;
      MulSrc<T, AXIS, Mul, false, (TABS > 0)> src{raw, P, outer, k0, mul};
      src.tab = atab;
      src.prep(tid % (P / 2));
      if constexpr (TSTORE && IsStoreField<Store>::value) {
        r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(work), src,
                                          RowStageSnk<T>{work, P}, tb, issue_next);
        store_tile(&dmap);
      } else if constexpr (TSTORE) {
        r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(work), src,
                                          RowStageValSnk<T, AXIS, Store>{work, P, outer, k0, st}, tb, issue_next);
        store_tile(&dmap);
      } else {
        r2r_tile<T, N, P / 2, NT, false>(ex, tid, kind, reinterpret_cast<Cx<T>*>(work), src,
                                          GlobSnk<T, AXIS, Store>{st, outer, k0}, tb, issue_next);
      }
    } else {
      // dense rows -> padded in-place tile (both sides contiguous in n); ks = 1
      // stages row[n + 1] at n and zero at the top
      if (ks == 0) {
        for (int e = tid; e < P * N; e += NT) {
          const int p = e / N, n = e - p * N;
          work[p * LD + n] = raw[e];
        }
      } else {
        for (int e = tid; e < P * N; e += NT) {
          const int p = e / N, n = e - p * N;
          work[p * LD + n] = n + 1 < N ? raw[e + 1] : T(0);
        }
      }
      __syncthreads();
      issue_next();
      r2r_tile_inplace<T, N, P / 2, NT>(ex, tid, kind, work, tb);
      // the tile's P rows lie in one x plane (P divides ny)
      const int row0 = t * P;
      const int i0 = row0 / g.ny, j0 = row0 - i0 * g.ny;
      if constexpr (IsStoreField<Store>::value) {
        constexpr int V = 16 / sizeof(T);   // 16-byte vector stores along z
        using VT = typename Vec4<T>::type;
        T* base = st.dst + size_t(row0) * N;
        for (int e = tid; e < P * N / V; e += NT) {
          const int p = (e * V) / N, n = e * V - p * N;
          VT v;
          T* vv = reinterpret_cast<T*>(&v);
#pragma unroll
          for (int u = 0; u < V; ++u) vv[u] = work[p * LD + n + u];
          *reinterpret_cast<VT*>(base + size_t(p) * N + n) = v;
        }
      } else {
        for (int e = tid; e < P * N; e += NT) {
          const int p = e / N, n = e - p * N;
          st(i0, j0 + p, n, work[p * LD + n]);
        }
      }
    }
    __syncthreads();   // the next tile's first stage overwrites `work`
  }
  if constexpr (TSTORE) {
    if (tid == 0) bulk_wait0();
  }
}

// ---------------------------------------------------------------------------
// Warp-tile x / y pass: the same tile transform as tma_pass_kernel, but every
// warp is an independent pipeline over its own tiles of PW = 2 G columns (G
// complex pencils: 2 in float, 1 in double) x all N rows: its own two landing
// buffers filled by its own TMA copies (a box PW columns wide, 16 bytes), its
// own mbarriers, its own work tile, staging rows and TMA stores, and warp-wide
// synchronisation only.  N <= 256 (one box along the axis).
// ---------------------------------------------------------------------------
template <typename T> constexpr int xyw_cols() { return sizeof(T) == 4 ? 4 : 2; }
constexpr int kXywWarps = 8;

template <typename T, int N>
struct XywLayout {
  static constexpr int PW = xyw_cols<T>(), G = PW / 2;
  static constexpr int RAW = PW * N;                                  // elements of one landing buffer
  static constexpr int WORK = ((PW * tile_ld(N) + 31) / 32) * 32;    // work tile elements (128-byte multiple)
  static constexpr size_t per_warp() { return size_t(2 * RAW + WORK) * sizeof(T); }
  static constexpr size_t smem_bytes() {
    return size_t(kXywWarps) * per_warp() + 2 * kXywWarps * 8 + 2 * N * sizeof(Cx<T>);
  }
  static_assert(RAW <= WORK, "the staging rows overlay the work tile");
};

template <typename T, int N, int AXIS, class Store, class Mul, class Mul2 = NoMul, bool TSTORE = false,
          int TABS = 0>
__global__ void __launch_bounds__(256, 2)
    tma_pass_warp_kernel(const __grid_constant__ CUtensorMap map, Geom g, int kind, Tables<T> tb, Store st,
                         int ntiles, int* err, uint32_t polls, int skip, Mul mul, int dc1, int dc2, Store st2,
                         Mul2 mul2, const __grid_constant__ CUtensorMap dmap,
                         const __grid_constant__ CUtensorMap dmap2) {
  static_assert(AXIS != 2 && N <= 256, "x / y passes of one box along the axis");
  using L = XywLayout<T, N>;
  constexpr int PW = L::PW, G = L::G, RAW = L::RAW;
  constexpr bool kDual = !std::is_same<Mul2, NoMul>::value;
  static_assert(!TSTORE || !kDual || IsStoreField<Store>::value, "dual passes stage plain fields");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  T* raw0 = reinterpret_cast<T*>(smem_raw + size_t(warp) * L::per_warp());
  T* raw1 = raw0 + RAW;
  T* work = raw1 + RAW;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + size_t(kXywWarps) * L::per_warp());
  uint64_t* bar = bars + 2 * warp;
  double* atab = reinterpret_cast<double*>(reinterpret_cast<Cx<T>*>(bars + 2 * kXywWarps) + 2 * N);
  {
    Cx<T>* rt = reinterpret_cast<Cx<T>*>(bars + 2 * kXywWarps);
    Cx<T>* qt = rt + N;
    for (int e = tid; e < N; e += 256) {
      rt[e] = tb.root[e];
      qt[e] = tb.quarter[e];
      if constexpr (TABS > 0) atab[e] = mul.axis_table(AXIS)[e];
      if constexpr (TABS > 1) atab[N + e] = mul2.axis_table(AXIS)[e];
    }
    tb.root = rt;
    tb.quarter = qt;
  }
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();   // tables and barriers ready: the only CTA-wide barrier
  const int w0 = int(blockIdx.x) * kXywWarps + warp, nw = int(gridDim.x) * kXywWarps;
  if (lane == 0) {
    if (w0 < ntiles && w0 != skip) tma_issue_tile<T, N, AXIS, PW>(&map, raw0, &bar[0], g, w0, dc1, dc2);
    if (w0 + nw < ntiles && w0 + nw != skip) tma_issue_tile<T, N, AXIS, PW>(&map, raw1, &bar[1], g, w0 + nw, dc1, dc2);
  }
  WarpExec ex;
  int it = 0;
  for (int t = w0; t < ntiles; t += nw, ++it) {
    const int b = it & 1;
    T* raw = b ? raw1 : raw0;
    const bool arrived = mbar_wait_bounded(&bar[b], (it >> 1) & 1, polls);
    if constexpr (TSTORE) {
      if (lane == 0) bulk_wait_read0();   // the previous tile's store has read the staging rows
    }
    if (!__all_sync(0xffffffffu, arrived)) {
      if (lane == 0) atomicExch(err, 1);
      drain_other(bar, b, it, t, nw, ntiles, skip, polls);
      break;
    }
    __syncwarp();
    const int t_next = t + 2 * nw;
    auto store_tile = [&](const CUtensorMap* dm) {
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        int c0, c1, c2;
        tile_origin<AXIS, PW>(g, t, c0, c1, c2);
        tma_store_3d(dm, work, c0, c1, c2);
        bulk_commit();
      }
    };
    auto issue_next = [&]() {
      if (lane == 0 && t_next < ntiles && t_next != skip) {
        fence_proxy_async_smem();
        tma_issue_tile<T, N, AXIS, PW>(&map, raw, &bar[b], g, t_next, dc1, dc2);
      }
    };
    const int kt = g.nz / PW;
    const int outer = t / kt, k0 = (t - outer * kt) * PW;
    MulSrc<T, AXIS, Mul, false, (TABS > 0)> src{raw, PW, outer, k0, mul};
    src.tab = atab;
    src.prep(lane % G);
    if constexpr (kDual) {
      if constexpr (TSTORE) {
        r2r_tile<T, N, G, 32, false>(ex, lane, kind, reinterpret_cast<Cx<T>*>(work), src, RowStageSnk<T>{work, PW}, tb);
        store_tile(&dmap);
        if (lane == 0) bulk_wait_read0();
      } else {
        r2r_tile<T, N, G, 32, false>(ex, lane, kind, reinterpret_cast<Cx<T>*>(work), src,
                                     GlobSnk<T, AXIS, Store>{st, outer, k0}, tb);
      }
      __syncwarp();   // the second transform rewrites the work tile
      MulSrc<T, AXIS, Mul2, false, (TABS > 1)> src2{raw, PW, outer, k0, mul2};
      src2.tab = atab + N;
      src2.prep(lane % G);
      if constexpr (TSTORE) {
        r2r_tile<T, N, G, 32, false>(ex, lane, kind, reinterpret_cast<Cx<T>*>(work), src2, RowStageSnk<T>{work, PW}, tb,
                                     issue_next);
        store_tile(&dmap2);
      } else {
        r2r_tile<T, N, G, 32, false>(ex, lane, kind, reinterpret_cast<Cx<T>*>(work), src2,
                                     GlobSnk<T, AXIS, Store>{st2, outer, k0}, tb, issue_next);
      }
    } else if constexpr (TSTORE && IsStoreField<Store>::value) {
      r2r_tile<T, N, G, 32, false>(ex, lane, kind, reinterpret_cast<Cx<T>*>(work), src, RowStageSnk<T>{work, PW}, tb,
                                   issue_next);
      store_tile(&dmap);
    } else if constexpr (TSTORE) {
      r2r_tile<T, N, G, 32, false>(ex, lane, kind, reinterpret_cast<Cx<T>*>(work), src,
                                   RowStageValSnk<T, AXIS, Store>{work, PW, outer, k0, st}, tb, issue_next);
      store_tile(&dmap);
    } else {
      r2r_tile<T, N, G, 32, false>(ex, lane, kind, reinterpret_cast<Cx<T>*>(work), src,
                                   GlobSnk<T, AXIS, Store>{st, outer, k0}, tb, issue_next);
    }
    __syncwarp();   // the next tile's first stage overwrites `work`
  }
  if constexpr (TSTORE) {
    if (lane == 0) bulk_wait0();
  }
}

template <typename T, int N, int P>
constexpr size_t tma_smem_bytes() {
  return size_t(2) * P * N * sizeof(T) + size_t(tma_work_elems<T, N, P>()) * sizeof(T) + 16 +
         2 * N * sizeof(Cx<T>);
}

// Pencils per tile.  z: rows per CTA; x/y: consecutive k (coalescing width).
template <typename T> constexpr int pass_pencils(int n) {
  return sizeof(T) == 8 ? (n >= 512 ? 8 : 16) : (n >= 512 ? 16 : 32);
}

template <typename T, int N, int AXIS, int P>
inline size_t pass_smem_bytes() {
  return size_t(P) * tile_ld(N) * sizeof(T);
}

template <typename T, int N, int AXIS, int P, class Load, class Store>
cudaError_t launch_pass_n(const Geom& g, int kind, Tables<T> tb, Load ld, Store st, cudaStream_t s) {
  const size_t smem = pass_smem_bytes<T, N, AXIS, P>();
  auto kern = axis_pass_kernel<T, N, AXIS, P, Load, Store>;
  static bool configured = false;   // per instantiation
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  int tiles;
  if (AXIS == 2) tiles = (g.nx * g.ny) / P;
  else if (AXIS == 1) tiles = g.nx * (g.nz / P);
  else tiles = g.ny * (g.nz / P);
  kern<<<tiles, pass_threads<T>(), smem, s>>>(g, kind, tb, ld, st);
  return cudaGetLastError();
}

// Plain field loads take the persistent TMA path when the tile fits a box
// (z: P divides ny and nz <= 256); `tma_err` receives wait timeouts.
struct TmaConfig {
  int* err = nullptr;     // device flag, nonzero after a timed-out wait
  uint32_t poll_limit = kTmaPollLimit;   // polls before a tile wait gives up
  int skip_tile = -1;     // fault injection: a tile whose copy is never issued
  const tc::Tables4* tc = nullptr;   // split-BF16 form: plain float x / y passes on the tensor cores
  // z passes of length 64..256 as warp tiles (tma_zpass_warp_kernel) rather
  // than CTA tiles, for float [0] and double [1] passes
  bool zwarp[2] = {false, true};
  // x [0] / y [1] passes as warp tiles (tma_pass_warp_kernel), float / double
  bool xywarp[2][2] = {{false, false}, {false, false}};
  int tc_axes = 3;        // with tc: the axes (bit 0 x, bit 1 y) that use it
  // z passes walk their tiles from the last x plane to the first, so that they
  // start on the rows the pass before them (a y pass or an elementwise stage,
  // both first plane to last) wrote last, which are still in L2
  bool zrev = true;
  int sms = 148;          // CTAs per SM x SMs bounds the persistent grid
  bool enabled = true;
};
inline TmaConfig& tma_config() {
  static thread_local TmaConfig c;
  return c;
}

// The warp-tile form of an x / y pass (tma_pass_warp_kernel).
template <typename T, int N, int AXIS, class Store, class Mul, class Mul2>
cudaError_t launch_tma_pass_warp(const Geom& g, int kind, Tables<T> tb, const T* src, Store st, cudaStream_t s,
                                 Mul mul, int dc1, int dc2, Store st2, Mul2 mul2) {
  using L = XywLayout<T, N>;
  constexpr int PW = L::PW;
  if (g.nz % PW != 0) return cudaErrorNotSupported;
  uint32_t box[3];
  if (AXIS == 1) { box[0] = PW; box[1] = N; box[2] = 1; }
  else { box[0] = PW; box[1] = 1; box[2] = N; }
  CUtensorMap map;
  if (!MapCache::get().lookup(&map, src, int(sizeof(T)), g.nx, g.ny, g.nz, AXIS, box)) return cudaErrorNotSupported;
  constexpr bool kStaged = IsStoreField<Store>::value || HasStageValue<Store>::value;
  constexpr bool TSTORE = kStaged;
  CUtensorMap dmap = map, dmap2 = map;
  if constexpr (TSTORE) {
    const T* dptr;
    if constexpr (IsStoreField<Store>::value) dptr = st.dst;
    else dptr = st.stage_dst();
    if (!MapCache::get().lookup(&dmap, dptr, int(sizeof(T)), g.nx, g.ny, g.nz, AXIS, box))
      return cudaErrorNotSupported;
    if constexpr (!std::is_same<Mul2, NoMul>::value) {
      if (!MapCache::get().lookup(&dmap2, st2.dst, int(sizeof(T)), g.nx, g.ny, g.nz, AXIS, box))
        return cudaErrorNotSupported;
    }
  }
  constexpr int TABS = row_tables<AXIS, Mul, Mul2>(L::smem_bytes(), N);
  const size_t smem = L::smem_bytes() + size_t(TABS) * N * sizeof(double);
  auto kern = tma_pass_warp_kernel<T, N, AXIS, Store, Mul, Mul2, TSTORE, TABS>;
  static int per_sm = 0;   // per instantiation: resident CTAs per SM
  if (per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 256, smem);
    if (e != cudaSuccess) return e;
    per_sm = n > 0 ? n : 1;
  }
  const int tiles = (AXIS == 1 ? g.nx : g.ny) * (g.nz / PW);
  const int full = per_sm * tma_config().sms;
  const int grid = tiles < full * kXywWarps ? (tiles + kXywWarps - 1) / kXywWarps : full;
  kern<<<grid, 256, smem, s>>>(map, g, kind, tb, st, tiles, tma_config().err, tma_config().poll_limit,
                               tma_config().skip_tile, mul, dc1, dc2, st2, mul2, dmap, dmap2);
  return cudaGetLastError();
}

template <typename T, int N, int AXIS, int P, class Store, class Mul = NoMul, class Mul2 = NoMul>
cudaError_t launch_tma_pass(const Geom& g, int kind, Tables<T> tb, const T* src, Store st, cudaStream_t s,
                            Mul mul = Mul(), int dc1 = 0, int dc2 = 0, int ks = 0, Store st2 = Store(),
                            Mul2 mul2 = Mul2()) {
  if constexpr (AXIS != 2 && N <= 256) {
    if (tma_config().xywarp[AXIS][sizeof(T) == 8]) {
      const cudaError_t e = launch_tma_pass_warp<T, N, AXIS>(g, kind, tb, src, st, s, mul, dc1, dc2, st2, mul2);
      if (e != cudaErrorNotSupported) return e;
    }
  }
  uint32_t box[3];
  constexpr int SUB = (N + 255) / 256;
  if (AXIS == 2) { box[0] = N; box[1] = P; box[2] = 1; }
  else if (AXIS == 1) { box[0] = P; box[1] = N / SUB; box[2] = 1; }
  else { box[0] = P; box[1] = 1; box[2] = N / SUB; }
  CUtensorMap map;
  if (!MapCache::get().lookup(&map, src, int(sizeof(T)), g.nx, g.ny, g.nz, AXIS, box)) return cudaErrorNotSupported;
  // plain field outputs of x / y passes leave through TMA stores (same box)
  constexpr bool kStaged = IsStoreField<Store>::value || HasStageValue<Store>::value;
  constexpr bool TSTORE = kStaged && AXIS != 2;
  CUtensorMap dmap = map, dmap2 = map;
  if constexpr (TSTORE) {
    const T* dptr;
    if constexpr (IsStoreField<Store>::value) dptr = st.dst;
    else dptr = st.stage_dst();
    if (!MapCache::get().lookup(&dmap, dptr, int(sizeof(T)), g.nx, g.ny, g.nz, AXIS, box))
      return cudaErrorNotSupported;
    if constexpr (!std::is_same<Mul2, NoMul>::value) {
      if (!MapCache::get().lookup(&dmap2, st2.dst, int(sizeof(T)), g.nx, g.ny, g.nz, AXIS, box))
        return cudaErrorNotSupported;
    }
  }
  constexpr int TABS = AXIS == 2 ? 0 : row_tables<AXIS, Mul, Mul2>(tma_smem_bytes<T, N, P>(), N);
  const size_t smem = tma_smem_bytes<T, N, P>() + size_t(TABS) * N * sizeof(double);
  // x / y passes (kFixedKind lengths) with the kind fixed at compile time:
  // every kind for plain passes, the inverse kinds for passes
  // with a spectral multiplier (which are always inverse transforms)
  using K = decltype(&tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS>);
  K kern = &tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS>;
  int slot = 0;
  if constexpr (kFixedKind<N> && AXIS != 2) {
    if constexpr (!Mul::kActive) {
      const K kk[4] = {&tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS, E10>,
                       &tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS, E01>,
                       &tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS, O10>,
                       &tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS, O01>};
      kern = kk[kind & 3];
      slot = 1 + (kind & 3);
    } else if (kind == E01) {
      kern = &tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS, E01>;
      slot = 1 + E01;
    } else if (kind == O01) {
      kern = &tma_pass_kernel<T, N, AXIS, P, Store, Mul, Mul2, TSTORE, TABS, O01>;
      slot = 1 + O01;
    }
  }
  static int per_sm_k[5] = {};   // per instantiation: resident CTAs per SM (runtime kind, then per fixed kind)
  int& per_sm = per_sm_k[slot];
  if (per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, tma_threads<T>(), smem);
    if (e != cudaSuccess) return e;
    per_sm = n > 0 ? n : 1;
  }
  int tiles;
  if (AXIS == 2) tiles = (g.nx * g.ny) / P;
  else if (AXIS == 1) tiles = g.nx * (g.nz / P);
  else tiles = g.ny * (g.nz / P);
  const int grid = tiles < per_sm * tma_config().sms ? tiles : per_sm * tma_config().sms;
  kern<<<grid, tma_threads<T>(), smem, s>>>(map, g, kind, tb, st, tiles, tma_config().err, tma_config().poll_limit,
                                             tma_config().skip_tile, mul, dc1, dc2, ks, st2, mul2, dmap, dmap2);
  return cudaGetLastError();
}

// Length of the transformed axis, its P, and the runtime switch over sizes.
template <typename T, int AXIS, class Load, class Store>
cudaError_t launch_pass(const Geom& g, int kind, Tables<T> tb, Load ld, Store st, cudaStream_t s) {
  const int n = AXIS == 0 ? g.nx : (AXIS == 1 ? g.ny : g.nz);
  // P pencils per tile must divide the tiled extent (rows nx*ny for z, nz for
  // x and y); 16 always does (validate_config), the wider tiles when they fit.
  const long extent = AXIS == 2 ? long(g.nx) * g.ny : long(g.nz);
#define QUASI_PASS_CASE(NN)                                                                   \
  case NN: {                                                                                  \
    constexpr int P = pass_pencils<T>(NN);                                                    \
    if (extent % P == 0) return launch_pass_n<T, NN, AXIS, P>(g, kind, tb, ld, st, s);        \
    return launch_pass_n<T, NN, AXIS, (P < 16 ? P : 16)>(g, kind, tb, ld, st, s);             \
  }
  switch (n) {
    QUASI_PASS_CASE(8)
    QUASI_PASS_CASE(16)
    QUASI_PASS_CASE(32)
    QUASI_PASS_CASE(64)
    QUASI_PASS_CASE(96)
    QUASI_PASS_CASE(128)
    QUASI_PASS_CASE(192)
    QUASI_PASS_CASE(256)
    QUASI_PASS_CASE(512)
    default: return cudaErrorInvalidValue;
  }
#undef QUASI_PASS_CASE
}

// z loads shifted by one along k: row[k + 1], zero at the top.
template <typename T>
struct ShiftKLoad {
  Geom g;
  const T* src;
  __device__ T operator()(int i, int j, int k) const { return k + 1 < g.nz ? src[lin(g, i, j, k + 1)] : T(0); }
};

// z loads shifted by one along k and scaled by -mk[k]: -mk[k] row[k + 1],
// zero at the top (the general-kernel form of the z pass with ks = 2).
template <typename T>
struct ShiftKMulLoad {
  Geom g;
  const T* src;
  const T* mk;
  __device__ T operator()(int i, int j, int k) const {
    return k + 1 < g.nz ? -mk[k] * src[lin(g, i, j, k + 1)] : T(0);
  }
};

// Plain field loads: the persistent TMA kernel when the tile fits a box,
// otherwise the general kernel above.  ks = 1 (z passes only) loads row[k + 1].
template <typename T, int AXIS, class Store>
cudaError_t launch_pass(const Geom& g, int kind, Tables<T> tb, LoadField<T> ld, Store st, cudaStream_t s,
                        int ks = 0) {
  const int n = AXIS == 0 ? g.nx : (AXIS == 1 ? g.ny : g.nz);
  const long extent = AXIS == 2 ? long(g.nx) * g.ny : long(g.nz);
  if constexpr (std::is_same<T, float>::value && AXIS != 2 && IsStoreField<Store>::value) {
    if (tma_config().tc && ((tma_config().tc_axes >> AXIS) & 1) && !ks) {
      const cudaError_t e = tc::launch_tc_pass(g.nx, g.ny, g.nz, AXIS, kind, *tma_config().tc, ld.src, st.dst,
                                               tma_config().err, tma_config().sms, s);
      if (e != cudaErrorNotSupported) return e;
    }
  }
  if (tma_config().enabled && tma_config().err) {
#define QUASI_TMA_CASE(NN)                                                                             \
    case NN: {                                                                                         \
      constexpr int P = pass_pencils<T>(NN);                                                           \
      const bool fits = extent % P == 0 && (AXIS != 2 || (NN <= 256 && g.ny % P == 0));                \
      if (fits) return launch_tma_pass<T, NN, AXIS, P>(g, kind, tb, ld.src, st, s, NoMul(), 0, 0, ks); \
      break;                                                                                           \
    }
    switch (n) {
      QUASI_TMA_CASE(16)
      QUASI_TMA_CASE(32)
      QUASI_TMA_CASE(64)
      QUASI_TMA_CASE(96)
      QUASI_TMA_CASE(128)
      QUASI_TMA_CASE(192)
      QUASI_TMA_CASE(256)
      QUASI_TMA_CASE(512)
      default: break;
    }
#undef QUASI_TMA_CASE
  }
  if (AXIS == 2 && ks) return launch_pass<T, AXIS, ShiftKLoad<T>, Store>(g, kind, tb, ShiftKLoad<T>{g, ld.src}, st, s);
  return launch_pass<T, AXIS, LoadField<T>, Store>(g, kind, tb, ld, st, s);
}

// x pass of an inverse transform whose input is mul(i,j,k) * src[i+di, j+dj, k]
// (di, dj in {0, 1}; rows shifted past the end read as zero).  Falls back to
// the general kernel with an equivalent loader when TMA is unavailable.
template <typename T, class Mul>
struct MulLoad {
  Geom g;
  const T* src;
  Mul mul;
  int di, dj;
  __device__ T operator()(int i, int j, int k) const {
    const int i1 = i + di, j1 = j + dj;
    if (i1 >= g.nx || j1 >= g.ny) return T(0);
    using M = decltype(mul(i, j, k));
    return T(M(src[lin(g, i1, j1, k)]) * mul(i, j, k));
  }
};

template <typename T, class Mul, class Store>
cudaError_t launch_mul_x_pass(const Geom& g, int kind, Tables<T> tb, const T* src, Mul mul, int di, int dj, Store st,
                              cudaStream_t s) {
  const long extent = g.nz;
  if (tma_config().enabled && tma_config().err) {
#define QUASI_TMA_CASE(NN)                                                                             \
    case NN: {                                                                                         \
      constexpr int P = pass_pencils<T>(NN);                                                           \
      if (extent % P == 0) return launch_tma_pass<T, NN, 0, P>(g, kind, tb, src, st, s, mul, dj, di);  \
      break;                                                                                           \
    }
    switch (g.nx) {
      QUASI_TMA_CASE(16)
      QUASI_TMA_CASE(32)
      QUASI_TMA_CASE(64)
      QUASI_TMA_CASE(96)
      QUASI_TMA_CASE(128)
      QUASI_TMA_CASE(192)
      QUASI_TMA_CASE(256)
      QUASI_TMA_CASE(512)
      default: break;
    }
#undef QUASI_TMA_CASE
  }
  return launch_pass<T, 0>(g, kind, tb, MulLoad<T, Mul>{g, src, mul, di, dj}, st, s);
}

// y pass whose input is mul(i,j,k) * src[i, j + 1, k] (the row past the end
// reads as zero): the y pass of a y gradient taken after a plain x pass.
template <typename T, class Mul, class Store>
cudaError_t launch_mul_y_pass(const Geom& g, int kind, Tables<T> tb, const T* src, Mul mul, Store st, cudaStream_t s) {
  const long extent = g.nz;
  if (tma_config().enabled && tma_config().err) {
#define QUASI_TMA_CASE(NN)                                                                            \
    case NN: {                                                                                        \
      constexpr int P = pass_pencils<T>(NN);                                                          \
      if (extent % P == 0) return launch_tma_pass<T, NN, 1, P>(g, kind, tb, src, st, s, mul, 1, 0);   \
      break;                                                                                          \
    }
    switch (g.ny) {
      QUASI_TMA_CASE(16)
      QUASI_TMA_CASE(32)
      QUASI_TMA_CASE(64)
      QUASI_TMA_CASE(96)
      QUASI_TMA_CASE(128)
      QUASI_TMA_CASE(192)
      QUASI_TMA_CASE(256)
      QUASI_TMA_CASE(512)
      default: break;
    }
#undef QUASI_TMA_CASE
  }
  return launch_pass<T, 1>(g, kind, tb, MulLoad<T, Mul>{g, src, mul, 0, 1}, st, s);
}

// Two x passes of the same shifted source with different multipliers, one tile
// load each (the general kernel runs them one after the other).
template <typename T, class Mul, class Mul2, class Store>
cudaError_t launch_mul_x_pass2(const Geom& g, int kind, Tables<T> tb, const T* src, Mul mul, Mul2 mul2, int di, int dj,
                               Store st, Store st2, cudaStream_t s) {
  const long extent = g.nz;
  if (tma_config().enabled && tma_config().err) {
#define QUASI_TMA_CASE(NN)                                                                              \
    case NN: {                                                                                          \
      constexpr int P = pass_pencils<T>(NN);                                                            \
      if (extent % P == 0)                                                                              \
        return launch_tma_pass<T, NN, 0, P, Store, Mul, Mul2>(g, kind, tb, src, st, s, mul, dj, di, 0, st2, \
                                                              mul2);                                    \
      break;                                                                                            \
    }
    switch (g.nx) {
      QUASI_TMA_CASE(16)
      QUASI_TMA_CASE(32)
      QUASI_TMA_CASE(64)
      QUASI_TMA_CASE(96)
      QUASI_TMA_CASE(128)
      QUASI_TMA_CASE(192)
      QUASI_TMA_CASE(256)
      QUASI_TMA_CASE(512)
      default: break;
    }
#undef QUASI_TMA_CASE
  }
  cudaError_t e = launch_pass<T, 0>(g, kind, tb, MulLoad<T, Mul>{g, src, mul, di, dj}, st, s);
  if (e != cudaSuccess) return e;
  return launch_pass<T, 0>(g, kind, tb, MulLoad<T, Mul2>{g, src, mul2, di, dj}, st2, s);
}

}  // namespace quasi
