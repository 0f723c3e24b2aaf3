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

#include "r2r_core.cuh"

namespace quasi {

struct DevExec {
  template <class R, class W, class Regs>
  __device__ __forceinline__ void phase2(R&& rd, W&& wr, int tid, Regs& regs) {
    rd(tid, regs);
    __syncthreads();
    wr(tid, regs);
    __syncthreads();
  }
};

struct Geom {
  int nx, ny, nz;
};

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

// Element e of a tile -> (pencil p, position n).  z tiles are P contiguous
// rows (n fastest); x/y tiles have P consecutive k (p fastest): either way
// neighbouring threads touch neighbouring addresses in global memory.
template <int AXIS, int P, int N>
__device__ __forceinline__ void tile_elem(int e, int& p, int& n) {
  if (AXIS == 2) { p = e / N; n = e - p * N; }
  else { n = e / P; p = e - n * P; }
}

// Threads per CTA: one radix-R_max butterfly per thread and pencil pair.
template <typename T> constexpr int pass_threads() { return sizeof(T) == 8 ? 128 : 256; }
// CTAs per SM the register allocation must allow (<= 128 registers/thread).
template <typename T> constexpr int pass_min_blocks() { return sizeof(T) == 8 ? 4 : 2; }

template <typename T, int N, int AXIS, int P, class Load, class Store>
__global__ void __launch_bounds__(pass_threads<T>(), pass_min_blocks<T>()) axis_pass_kernel(Geom g, int kind, Tables<T> tb, Load ld,
                                                                      Store st) {
  constexpr int NT = pass_threads<T>();
  constexpr int LD = tile_ld(N);
  constexpr int E = P * N;
  constexpr int PER = (E + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* buf = reinterpret_cast<T*>(smem_raw);
  const int tile = blockIdx.x;
  const int tid = threadIdx.x;
  // loads go out in batches of B per thread (B * NT * sizeof(T) bytes in
  // flight per CTA) before any of them is consumed
  constexpr int B = PER < 16 ? PER : 16;
#pragma unroll
  for (int c0 = 0; c0 < PER; c0 += B) {
    T v[B];
#pragma unroll
    for (int c = 0; c < B; ++c) {
      const int e = tid + (c0 + c) * NT;
      if ((E % NT == 0 && PER % B == 0) || (c0 + c < PER && e < E)) {
        int p, n, i, j, k;
        tile_elem<AXIS, P, N>(e, p, n);
        tile_coords<AXIS>(g, tile, P, p, n, i, j, k);
        v[c] = ld(i, j, k);
      }
    }
#pragma unroll
    for (int c = 0; c < B; ++c) {
      const int e = tid + (c0 + c) * NT;
      if ((E % NT == 0 && PER % B == 0) || (c0 + c < PER && e < E)) {
        int p, n;
        tile_elem<AXIS, P, N>(e, p, n);
        buf[p * LD + n] = v[c];
      }
    }
  }
  __syncthreads();
  DevExec ex;
  r2r_tile_inplace<T, N, P / 2, NT>(ex, tid, kind, buf, tb);
#pragma unroll
  for (int c = 0; c < PER; ++c) {
    const int e = tid + c * NT;
    if (E % NT == 0 || e < E) {
      int p, n, i, j, k;
      tile_elem<AXIS, P, N>(e, p, n);
      tile_coords<AXIS>(g, tile, P, p, n, i, j, k);
      st(i, j, k, buf[p * LD + n]);
    }
  }
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
};

template <typename T>
struct StoreField {
  Geom g;
  T* dst;
  __device__ void operator()(int i, int j, int k, T v) const { dst[lin(g, i, j, k)] = v; }
};

template <typename T>
struct ScaleStore {
  Geom g;
  T* dst;
  T s;
  __device__ void operator()(int i, int j, int k, T v) const { dst[lin(g, i, j, k)] = v * s; }
};

}  // namespace quasi
