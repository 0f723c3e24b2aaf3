// Tensor-memory-accelerator (TMA) tile loads for the axis passes: tensor maps
// built on the host through the driver entry point, and the device-side
// mbarrier / cp.async.bulk.tensor primitives (inline PTX, sm_90+ / sm_100a).
// Loads and stores, one CTA each: no cluster multicast anywhere.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>

namespace quasi {

// ---------------------------------------------------------------------------
// Device side
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each poll itself suspends the
// thread for a hardware-defined interval) and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// Tile stores: shared memory -> global through a tensor map (bulk groups,
// committed and awaited by the issuing thread).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src))
      : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the smem sources of all committed bulk stores have been read
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// all committed bulk stores are complete
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Host side: one tensor map per (field, axis) over the field as a 3-D tensor
// (nz, ny, nx) (innermost first), box = the pass's tile (<= 256 per dim).
// ---------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// box: per-axis box extents (k, j, i).  Returns false if the map cannot be built.
inline bool make_field_map(CUtensorMap* map, const void* base, int elem, int nx, int ny, int nz, const uint32_t box[3]) {
  EncodeTiledFn fn = encode_tiled_fn();
  if (!fn) return false;
  const cuuint64_t dims[3] = {cuuint64_t(nz), cuuint64_t(ny), cuuint64_t(nx)};
  const cuuint64_t strides[2] = {cuuint64_t(nz) * elem, cuuint64_t(ny) * nz * elem};
  const cuuint32_t bx[3] = {box[0], box[1], box[2]};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUtensorMapDataType dt = elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r = fn(map, dt, 3, const_cast<void*>(base), dims, strides, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Process-wide cache: maps are plain 128-byte descriptors passed by value as
// __grid_constant__ kernel parameters (captured into the step graphs).
class MapCache {
 public:
  static MapCache& get() {
    static MapCache c;
    return c;
  }
  bool lookup(CUtensorMap* out, const void* base, int elem, int nx, int ny, int nz, int axis, const uint32_t box[3]) {
    int dev = 0;
    cudaGetDevice(&dev);
    auto key = std::make_tuple(dev, base, elem, nx, ny, nz, axis, box[0], box[1], box[2]);
    std::lock_guard<std::mutex> lk(mu_);
    auto it = maps_.find(key);
    if (it != maps_.end()) {
      *out = it->second;
      return true;
    }
    CUtensorMap m;
    if (!make_field_map(&m, base, elem, nx, ny, nz, box)) return false;
    maps_.emplace(key, m);
    *out = m;
    return true;
  }
  // a freed field must not be found again under a reused address
  void forget(const void* lo, const void* hi) {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto it = maps_.begin(); it != maps_.end();) {
      const void* b = std::get<1>(it->first);
      if (b >= lo && b < hi) it = maps_.erase(it);
      else ++it;
    }
  }

 private:
  std::mutex mu_;
  std::map<std::tuple<int, const void*, int, int, int, int, int, uint32_t, uint32_t, uint32_t>, CUtensorMap> maps_;
};

}  // namespace quasi
