// The y and z transforms of a field in ONE pass: a thread-block cluster of
// C CTAs owns one x plane (ny x nz) at a time.
//
//   1. each CTA receives ny/C = R rows of the plane by TMA (box nz x R) and
//      transforms them along z in place (padded shared tile);
//   2. cluster barrier; each CTA pushes its rows, split by column block, into
//      every CTA's interleaved [j][Q] column tile through distributed shared
//      memory (adjacent k pencils are one complex value there);
//   3. cluster barrier; each CTA transforms its columns along y and stores
//      them (coalesced rows of Q elements).
// Planes are walked persistently with the next plane's rows prefetched by
// TMA.  A 3-D transform is then this pass plus one x pass: two trips through
// HBM instead of three.  Loads only; no cluster multicast.
#pragma once
#include <cooperative_groups.h>

#include "r2r_pass.cuh"

namespace quasi {

namespace cg = cooperative_groups;

template <typename T, int NY, int NZ, int C>
struct YZShape {
  static constexpr int R = NY / C;   // rows per CTA (z phase)
  static constexpr int Q = NZ / C;   // columns per CTA (y phase)
  static constexpr int RAW = R * NZ;  // == NY * Q
  static constexpr int WORK = (R * tile_ld(NZ) > Q * tile_ld(NY) ? R * tile_ld(NZ) : Q * tile_ld(NY));
  static constexpr int WORK_PAD = ((WORK + 31) / 32) * 32;
  static constexpr size_t bytes() { return (size_t(2) * RAW + WORK_PAD) * sizeof(T) + 64; }
  static_assert(R % 2 == 0 && Q % 2 == 0, "R and Q must be even (pencil pairs)");
};

template <typename T, int NY, int NZ, int C>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1)
    yz_plane_kernel(const __grid_constant__ CUtensorMap map, Geom g, int kind_y, int kind_z, Tables<T> tby,
                    Tables<T> tbz, StoreField<T> st, int* err) {
  using S = YZShape<T, NY, NZ, C>;
  constexpr int NT = 256;
  constexpr int R = S::R, Q = S::Q;
  constexpr int LDZ = tile_ld(NZ);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* raw0 = reinterpret_cast<T*>(smem_raw);
  T* raw1 = raw0 + S::RAW;
  T* work = raw1 + S::RAW;
  uint64_t* bar = reinterpret_cast<uint64_t*>(work + S::WORK_PAD);
  int* vote = reinterpret_cast<int*>(bar + 2);
  cg::cluster_group cluster = cg::this_cluster();
  const int c = int(cluster.block_rank());
  const int nclusters = gridDim.x / C;
  const int cid = blockIdx.x / C;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](T* dst, uint64_t* b, int plane) {
    mbar_expect_tx(b, uint32_t(S::RAW * sizeof(T)));
    tma_load_3d(dst, &map, b, 0, c * R, plane);
  };
  if (tid == 0) {
    if (cid < g.nx) issue(raw0, &bar[0], cid);
    if (cid + nclusters < g.nx) issue(raw1, &bar[1], cid + nclusters);
  }
  DevExec ex;
  int it = 0;
  for (int plane = cid; plane < g.nx; plane += nclusters, ++it) {
    const int b = it & 1;
    T* raw = b ? raw1 : raw0;
    const bool arrived = mbar_wait_bounded(&bar[b], (it >> 1) & 1, kTmaPollLimit);
    const int ok = __syncthreads_and(arrived);
    // 1. rows -> padded tile, transform along z
    for (int e = tid; e < S::RAW; e += NT) {
      const int r = e / NZ, n = e - r * NZ;
      work[r * LDZ + n] = raw[e];
    }
    __syncthreads();
    r2r_tile_inplace<T, NZ, R / 2, NT>(ex, tid, kind_z, work, tbz);
    // the cluster leaves together if any CTA's tile never arrived
    if (tid == 0) *vote = ok;
    cluster.sync();
    int all_ok = 1;
    for (int q = 0; q < C; ++q) all_ok &= *cluster.map_shared_rank(vote, q);
    if (!all_ok) {
      if (tid == 0 && !ok) atomicExch(err, 1);
      break;
    }
    // 2. push this CTA's rows into every CTA's column tile col[j][kk] (the
    //    peer's raw buffer, free since the barrier above): remote stores do
    //    not stall, and consecutive threads write consecutive peer addresses
    T* col = raw;
    for (int e = tid; e < S::RAW; e += NT) {
      const int r = e / NZ, n = e - r * NZ;
      const int dst = n / Q, kk = n - dst * Q;
      T* peer = cluster.map_shared_rank(col, dst);
      peer[(c * R + r) * Q + kk] = work[r * LDZ + n];
    }
    cluster.sync();   // every column tile complete; `work` may be reused
    // 3. transform the columns along y; the raw buffer is recycled for the
    //    plane after next as soon as the first stage has read it
    const int next = plane + 2 * nclusters;
    auto issue_next = [&]() {
      if (tid == 0 && next < g.nx) {
        fence_proxy_async_smem();
        issue(raw, &bar[b], next);
      }
    };
    r2r_tile<T, NY, Q / 2, NT, false>(ex, tid, kind_y, reinterpret_cast<Cx<T>*>(work), RawSrc<T>{col, Q},
                                       GlobSnk<T, 1, StoreField<T>>{st, plane, c * Q}, tby, issue_next);
    __syncthreads();
  }
  cluster.sync();   // no CTA leaves while a peer may still read its tile
}

// Cluster size for a plane: the smallest C (<= 8) whose per-CTA slab fits
// 32 KB (FP32) / 64 KB (FP64) with R and Q even; 0 if none.
template <typename T, int NY, int NZ>
constexpr int yz_cluster_size() {
  const size_t plane = size_t(NY) * NZ * sizeof(T);
  const size_t cap = sizeof(T) == 8 ? 65536 : 32768;
  for (int c = 1; c <= 8; c *= 2)
    if (NY % (2 * c) == 0 && NZ % (2 * c) == 0 && plane / c <= cap) return c;
  return 0;
}

template <typename T, int NY, int NZ>
cudaError_t launch_yz_n(const Geom& g, int kind_y, int kind_z, Tables<T> tby, Tables<T> tbz, const T* src, T* dst,
                        cudaStream_t s) {
  constexpr int C = yz_cluster_size<T, NY, NZ>();
  if constexpr (C == 0) {
    return cudaErrorNotSupported;
  } else {
    using S = YZShape<T, NY, NZ, C>;
    const uint32_t box[3] = {uint32_t(NZ), uint32_t(S::R), 1};
    CUtensorMap map;
    if (!MapCache::get().lookup(&map, src, int(sizeof(T)), g.nx, g.ny, g.nz, 3, box)) return cudaErrorNotSupported;
    auto kern = yz_plane_kernel<T, NY, NZ, C>;
    const size_t smem = S::bytes();
    static bool configured = false;
    if (!configured) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess) return e;
      configured = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // persistent grid: as many clusters as the GPCs hold at once (a cluster
    // must fit one GPC, so this is below SMs x CTAs-per-SM / C)
    static int resident = 0;
    if (resident == 0) {
      cfg.gridDim = dim3(C);
      cudaError_t e = cudaOccupancyMaxActiveClusters(&resident, kern, &cfg);
      if (e != cudaSuccess) return e;
      if (resident < 1) return cudaErrorNotSupported;
    }
    int clusters = resident < g.nx ? resident : g.nx;
    cfg.gridDim = dim3(clusters * C);
    return cudaLaunchKernelEx(&cfg, kern, map, g, kind_y, kind_z, tby, tbz, StoreField<T>{g, dst},
                              tma_config().err);
  }
}

// y and z transforms of src -> dst in one pass when the plane shape is one of
// the instantiated ones; cudaErrorNotSupported otherwise (caller falls back).
template <typename T>
cudaError_t launch_yz(const Geom& g, int kind_y, int kind_z, Tables<T> tby, Tables<T> tbz, const T* src, T* dst,
                      cudaStream_t s) {
  if (!tma_config().enabled || !tma_config().err || !tma_config().yz) return cudaErrorNotSupported;
#define QUASI_YZ(A, B) \
  if (g.ny == A && g.nz == B) return launch_yz_n<T, A, B>(g, kind_y, kind_z, tby, tbz, src, dst, s);
  QUASI_YZ(256, 256)
  QUASI_YZ(128, 128)
  QUASI_YZ(128, 256)
  QUASI_YZ(64, 128)
  QUASI_YZ(96, 192)
  QUASI_YZ(32, 64)
  QUASI_YZ(16, 32)
#undef QUASI_YZ
  return cudaErrorNotSupported;
}

}  // namespace quasi
