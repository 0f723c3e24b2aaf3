// Tensor-core form of an x or y axis pass (N = 256): the r2r transform along
// the axis as a dense contraction with the FFTW kind's matrix on the sm_100a
// tensor cores (tcgen05.mma, accumulators in tensor memory), with split-BF16
// operands: each float operand is hi + lo (two BF16 values), and
//   A x ~= A_hi x_hi + A_hi x_lo + A_lo x_hi      (FP32 accumulation)
// which keeps ~17 of float's 24 significant bits per product.
//
// Even/odd folding halves the work.  For the forward kinds (REDFT10, RODFT10)
// the input pairs x_m +- x_{N-1-m} feed two N/2 x N/2 matrices whose outputs
// are the even and odd rows y_{2p}, y_{2p+1}; for the inverse kinds (REDFT01,
// RODFT01) the even and odd input rows feed two matrices E, O and the outputs
// are y_k = E_k + O_k, y_{N-1-k} = E_k - O_k (k < N/2).  The matrices are
// FFTW's published definitions (the kinds of quasi.cpp:449-495), built on the
// host in long double.
//
// One CTA per SM, persistent over column tiles of 64 contiguous floats:
//   A (the four folded half-matrices hi/lo, 128 KB) stays in shared memory,
//     K-major with the 128-byte swizzle, loaded once;
//   B (this tile's folded input, hi/lo, 64 KB) is written by the threads from
//     registers (the tile was loaded one iteration ahead), MN-major with the
//     128-byte swizzle, so a thread's float4 from global memory lands as one
//     8-byte store;
//   one thread issues 2 x 8 x 3 MMAs of 128 x 64 x 16 into one of two
//     accumulator sets in tensor memory (2 x 2 x 64 columns) and commits them
//     to an mbarrier; meanwhile the threads load the next tile and read the
//     previous tile's accumulators (tcgen05.ld) and store its outputs.
// No cluster, no multicast: one CTA's own shared memory and tensor memory.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "r2r_core.cuh"
#ifdef __CUDACC__
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "tma.cuh"
#endif

namespace quasi {

namespace tc {

constexpr int kN = 256;            // transform length
constexpr int kH = kN / 2;         // folded length: MMA M and K
constexpr int kCols = 64;          // column tile: MMA N
constexpr int kThreads = 256;
constexpr int kAtom = kH * 128;    // one K-major swizzle atom: 128 rows x 128 bytes
constexpr int kMat = 2 * kAtom;    // one 128 x 128 BF16 matrix (two atoms along K) = 32 KB
constexpr int kBMat = kH * kCols * 2;   // one 128 x 64 BF16 operand = 16 KB
constexpr int kSmemA = 4 * kMat;        // even hi, even lo, odd hi, odd lo
constexpr int kSmemB = 4 * kBMat;
constexpr int kTmemCols = 256;          // 2 sets x (even, odd) x 64 columns
constexpr size_t kSmemBytes = size_t(kSmemA) + kSmemB + 1024 /* alignment */ + 64;
constexpr uint32_t kPollLimit = 1u << 24;

// Byte offset of element (row r, k) in a K-major 128-byte-swizzled matrix of
// 128 rows and 128 k (BF16): atom k/64, 8-row groups 1024 bytes apart, rows
// 128 bytes apart, the 16-byte chunk index XOR-ed with the row within its group.
QHD constexpr int a_offset(int r, int k) {
  return (k >> 6) * kAtom + (r >> 3) * 1024 + (r & 7) * 128 + ((((k & 63) >> 3) ^ (r & 7)) << 4) + (k & 7) * 2;
}
// Byte offset of element (k, n) in an MN-major 128-byte-swizzled operand of
// 128 k x 64 n (BF16): 8-k groups 1024 bytes apart, k rows 128 bytes apart,
// the 16-byte chunk (8 n) XOR-ed with the k row within its group.
QHD constexpr int b_offset(int k, int n) {
  return (k >> 3) * 1024 + (k & 7) * 128 + (((n >> 3) ^ (k & 7)) << 4) + (n & 7) * 2;
}

// Shared-memory matrix descriptor (tcgen05 "UMMA" format): start address,
// leading and stride byte offsets in 16-byte units, version 1, 128-byte
// swizzle (layout type 2).
QHD constexpr uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46) | (uint64_t(2) << 61);
}
// Instruction descriptor of kind::f16: BF16 A (K-major) and B (MN-major),
// FP32 accumulator, M = 128, N = 64.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | (uint32_t(kCols >> 3) << 17) |
                            (uint32_t(kH >> 4) << 24);

// Round a float to BF16 (nearest, ties to even) on the host; returns the bits.
inline uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return uint16_t(u >> 16);
}
inline float bf16_value(uint16_t b) {
  const uint32_t u = uint32_t(b) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// The four swizzled half-matrices of `kind` (even hi, even lo, odd hi, odd
// lo) as one 128 KB image of the shared-memory operand A.
inline std::vector<uint16_t> folded_matrices(int kind) {
  const long double pi = 3.14159265358979323846264338327950288L;
  const int N = kN, H = kH;
  std::vector<uint16_t> img(kSmemA / 2, 0);
  for (int p = 0; p < H; ++p)
    for (int m = 0; m < H; ++m) {
      long double e, o;
      if (kind == E10) {          // rows 2p <- x_m + x_{N-1-m}, 2p+1 <- x_m - x_{N-1-m}
        e = 2 * std::cos(pi * (2 * p) * (2 * m + 1) / (2 * N));
        o = 2 * std::cos(pi * (2 * p + 1) * (2 * m + 1) / (2 * N));
      } else if (kind == O10) {
        e = 2 * std::sin(pi * (2 * p + 1) * (2 * m + 1) / (2 * N));
        o = 2 * std::sin(pi * (2 * p + 2) * (2 * m + 1) / (2 * N));
      } else if (kind == E01) {   // E from the even rows x_{2m}, O from the odd rows
        e = (m == 0 ? 1 : 2) * std::cos(pi * (2 * m) * (2 * p + 1) / (2 * N));
        o = 2 * std::cos(pi * (2 * m + 1) * (2 * p + 1) / (2 * N));
      } else {                    // O01: x_{N-1} enters with weight 1
        e = 2 * std::sin(pi * (2 * m + 1) * (2 * p + 1) / (2 * N));
        o = (m == H - 1 ? 1 : 2) * std::sin(pi * (2 * m + 2) * (2 * p + 1) / (2 * N));
      }
      const long double v[2] = {e, o};
      for (int s = 0; s < 2; ++s) {
        const uint16_t hi = bf16_bits(float(v[s]));
        const uint16_t lo = bf16_bits(float(v[s] - (long double)bf16_value(hi)));
        img[(s * 2 * kMat + a_offset(p, m)) / 2] = hi;
        img[(s * 2 * kMat + kMat + a_offset(p, m)) / 2] = lo;
      }
    }
  return img;
}

#ifdef __CUDACC__
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Tile geometry: the transform axis has stride `axis_stride` (elements); a
// batch holds `cols` contiguous columns (x pass: ny*nz columns, one batch;
// y pass: nz columns, nx batches `batch_stride` apart).  Tile t covers 64
// columns of one batch.
struct TcGeom {
  size_t axis_stride, batch_stride;
  int tiles_per_batch, ntiles;
};

template <bool FWD>
struct TcTile {
  static constexpr int kPairs = (kH * kCols / 4) / kThreads;   // float4 pairs per thread (8)
  float4 a[kPairs], b[kPairs];
  // rows of pair m: forward (m, N-1-m), inverse (2m, 2m+1)
  __device__ static int row_a(int m) { return FWD ? m : 2 * m; }
  __device__ static int row_b(int m) { return FWD ? kN - 1 - m : 2 * m + 1; }
  __device__ void load(const float* src, size_t base, const TcGeom& gm, int tid) {
#pragma unroll
    for (int r = 0; r < kPairs; ++r) {
      const int P = tid + kThreads * r, m = P >> 4, q = P & 15;
      a[r] = __ldg(reinterpret_cast<const float4*>(src + base + size_t(row_a(m)) * gm.axis_stride) + q);
      b[r] = __ldg(reinterpret_cast<const float4*>(src + base + size_t(row_b(m)) * gm.axis_stride) + q);
    }
  }
};

__device__ __forceinline__ void split_store(unsigned char* hi, unsigned char* lo, int off, float v0, float v1,
                                            float v2, float v3) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1), h2 = __float2bfloat16_rn(v2),
                      h3 = __float2bfloat16_rn(v3);
  const __nv_bfloat16 l0 = __float2bfloat16_rn(v0 - __bfloat162float(h0)),
                      l1 = __float2bfloat16_rn(v1 - __bfloat162float(h1)),
                      l2 = __float2bfloat16_rn(v2 - __bfloat162float(h2)),
                      l3 = __float2bfloat16_rn(v3 - __bfloat162float(h3));
  __nv_bfloat162 hv[2] = {__halves2bfloat162(h0, h1), __halves2bfloat162(h2, h3)};
  __nv_bfloat162 lv[2] = {__halves2bfloat162(l0, l1), __halves2bfloat162(l2, l3)};
  *reinterpret_cast<uint2*>(hi + off) = *reinterpret_cast<const uint2*>(hv);
  *reinterpret_cast<uint2*>(lo + off) = *reinterpret_cast<const uint2*>(lv);
}

// Outputs of one tile from accumulator set `sset`: warp w reads the lanes of
// its sub-partition (w % 4) and 32 of the 64 columns (w / 4), and writes two
// output rows per lane (forward: 2p, 2p + 1; inverse: p, N-1-p).
template <bool FWD>
__device__ __forceinline__ void tc_epilogue(float* dst, size_t tbase, const TcGeom& gm, uint32_t tmem, uint32_t sset,
                                            int warp, int lane) {
  const int sp = warp & 3, ch = warp >> 2;
  const int p = sp * 32 + lane;
  float e[32], o[32];
  const uint32_t ta = tmem + (uint32_t(sp * 32) << 16) + sset + uint32_t(ch * 32);
  tmem_ld32(ta, e);
  tmem_ld32(ta + 64, o);
  const size_t base = tbase + size_t(ch * 32);
  float* r0 = dst + base + size_t(FWD ? 2 * p : p) * gm.axis_stride;
  float* r1 = dst + base + size_t(FWD ? 2 * p + 1 : kN - 1 - p) * gm.axis_stride;
#pragma unroll
  for (int c = 0; c < 32; c += 4) {
    float4 u, w;
    if (FWD) {
      u = make_float4(e[c], e[c + 1], e[c + 2], e[c + 3]);
      w = make_float4(o[c], o[c + 1], o[c + 2], o[c + 3]);
    } else {
      u = make_float4(e[c] + o[c], e[c + 1] + o[c + 1], e[c + 2] + o[c + 2], e[c + 3] + o[c + 3]);
      w = make_float4(e[c] - o[c], e[c + 1] - o[c + 1], e[c + 2] - o[c + 2], e[c + 3] - o[c + 3]);
    }
    *reinterpret_cast<float4*>(r0 + c) = u;
    *reinterpret_cast<float4*>(r1 + c) = w;
  }
}

// One axis pass src -> dst (may alias: every tile's columns are read before
// any of its outputs are written, and tiles are disjoint).  `amat`: the 128 KB
// operand image of the kind (folded_matrices).  A timed-out MMA wait sets *err.
template <bool FWD>
__global__ void __launch_bounds__(kThreads, 1)
    tc_pass_kernel(const float* src, float* dst, const uint4* amat, TcGeom gm, int* err) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sa = smem;                  // A: even hi, even lo, odd hi, odd lo
  unsigned char* sb = smem + kSmemA;         // B: even hi, even lo, odd hi, odd lo
  uint64_t* bar = reinterpret_cast<uint64_t*>(sb + kSmemB);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // A once per CTA (L2-resident after the first CTAs)
  for (int i = tid; i < kSmemA / 16; i += kThreads) reinterpret_cast<uint4*>(sa)[i] = __ldg(amat + i);
  if (warp == 0) tmem_alloc(tslot, kTmemCols);
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t sa_u = smem_u32(sa), sb_u = smem_u32(sb);

  TcTile<FWD> cur;
  auto tile_base = [&](int t) {
    const int b = t / gm.tiles_per_batch, c = t - b * gm.tiles_per_batch;
    return size_t(b) * gm.batch_stride + size_t(c) * kCols;
  };
  int t = blockIdx.x;
  if (t < gm.ntiles) cur.load(src, tile_base(t), gm, tid);
  bool ok = true;
  int it = 0, prev_t = -1;
  for (; t < gm.ntiles; t += gridDim.x, ++it) {
    // this tile's folded input into B (hi / lo); B is free: the previous
    // tile's MMAs completed before the end of the last iteration
#pragma unroll
    for (int r = 0; r < TcTile<FWD>::kPairs; ++r) {
      const int P = tid + kThreads * r, m = P >> 4, q = P & 15;
      const float4 x = cur.a[r], y = cur.b[r];
      float4 s, d;
      if (FWD) {
        s = make_float4(x.x + y.x, x.y + y.y, x.z + y.z, x.w + y.w);
        d = make_float4(x.x - y.x, x.y - y.y, x.z - y.z, x.w - y.w);
      } else {
        s = x;
        d = y;
      }
      const int off = b_offset(m, 4 * q);
      split_store(sb, sb + kBMat, off, s.x, s.y, s.z, s.w);
      split_store(sb + 2 * kBMat, sb + 3 * kBMat, off, d.x, d.y, d.z, d.w);
    }
    fence_proxy_async_smem();
    __syncthreads();
    const uint32_t set = uint32_t(it & 1) * 128;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int h = 0; h < 2; ++h) {          // even, odd
        const uint32_t d_tmem = tmem + set + uint32_t(h) * 64;
        const uint32_t a0 = sa_u + uint32_t(h) * 2 * kMat, b0 = sb_u + uint32_t(h) * 2 * kBMat;
#pragma unroll
        for (int ks = 0; ks < kH / 16; ++ks) {
          const uint32_t aoff = uint32_t((ks >> 2) * kAtom + (ks & 3) * 32), boff = uint32_t(ks * 2048);
          const uint64_t ahi = smem_desc(a0 + aoff, 16, 1024), alo = smem_desc(a0 + kMat + aoff, 16, 1024);
          const uint64_t bhi = smem_desc(b0 + boff, kBMat, 1024), blo = smem_desc(b0 + kBMat + boff, kBMat, 1024);
          mma_bf16(d_tmem, ahi, blo, kIdesc, ks > 0);
          mma_bf16(d_tmem, alo, bhi, kIdesc, 1);
          mma_bf16(d_tmem, ahi, bhi, kIdesc, 1);
        }
      }
      mma_commit(bar);
    }
    // the next tile's loads are in flight while the MMAs run and the previous
    // tile's outputs leave
    const int tn = t + int(gridDim.x);
    if (tn < gm.ntiles) cur.load(src, tile_base(tn), gm, tid);
    if (prev_t >= 0) tc_epilogue<FWD>(dst, tile_base(prev_t), gm, tmem, set ^ 128u, warp, lane);
    tc_fence_before();
    // this tile's MMAs done: B may be rewritten, its accumulators are ready
    const bool arrived = mbar_wait_bounded(bar, uint32_t(it & 1), kPollLimit);
    if (!__syncthreads_and(arrived)) {
      if (tid == 0) atomicExch(err, 1);
      ok = false;
      break;
    }
    tc_fence_after();
    prev_t = t;
  }
  // the last tile's outputs (its accumulators: the last iteration's set)
  if (ok && prev_t >= 0) tc_epilogue<FWD>(dst, tile_base(prev_t), gm, tmem, uint32_t((it - 1) & 1) * 128, warp, lane);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// Device images of operand A for the four kinds (one 128 KB image each).
struct Tables4 {
  const uint4* a[4] = {nullptr, nullptr, nullptr, nullptr};
};

inline cudaError_t upload_tables(Tables4& t, void** owned) {
  cudaError_t e = cudaMalloc(owned, size_t(4) * kSmemA);
  if (e != cudaSuccess) return e;
  for (int k = 0; k < 4; ++k) {
    const std::vector<uint16_t> img = folded_matrices(k);
    char* d = static_cast<char*>(*owned) + size_t(k) * kSmemA;
    if ((e = cudaMemcpy(d, img.data(), kSmemA, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    t.a[k] = reinterpret_cast<const uint4*>(d);
  }
  return cudaSuccess;
}

// x (axis 0) or y (axis 1) pass of a float field with N = 256 along the axis
// on the tensor cores; cudaErrorNotSupported for other shapes (the caller
// takes the FFT pass).  src and dst may alias.
inline cudaError_t launch_tc_pass(int nx, int ny, int nz, int axis, int kind, const Tables4& tt, const float* src,
                                  float* dst, int* err, int sms, cudaStream_t s) {
  TcGeom gm{};
  if (axis == 0) {
    if (nx != kN || (size_t(ny) * nz) % kCols) return cudaErrorNotSupported;
    gm.axis_stride = size_t(ny) * nz;
    gm.batch_stride = 0;
    gm.tiles_per_batch = int(size_t(ny) * nz / kCols);
    gm.ntiles = gm.tiles_per_batch;
  } else if (axis == 1) {
    if (ny != kN || nz % kCols) return cudaErrorNotSupported;
    gm.axis_stride = size_t(nz);
    gm.batch_stride = size_t(ny) * nz;
    gm.tiles_per_batch = nz / kCols;
    gm.ntiles = nx * gm.tiles_per_batch;
  } else {
    return cudaErrorNotSupported;
  }
  if (kind < 0 || kind > 3 || !tt.a[kind]) return cudaErrorInvalidValue;
  const bool fwd = is_forward(kind);
  auto kern = fwd ? tc_pass_kernel<true> : tc_pass_kernel<false>;
  static bool configured[2] = {false, false};
  if (!configured[fwd]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes));
    if (e != cudaSuccess) return e;
    configured[fwd] = true;
  }
  const int grid = gm.ntiles < sms ? gm.ntiles : sms;
  kern<<<grid, kThreads, kSmemBytes, s>>>(src, dst, tt.a[kind], gm, err);
  return cudaGetLastError();
}
#endif

}  // namespace tc
}  // namespace quasi
