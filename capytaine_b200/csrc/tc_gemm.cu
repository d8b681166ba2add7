// Complex trailing update on the 5th-generation tensor cores (tcgen05, TF32
// inputs, FP32 accumulation in tensor memory).
//
// The mixed-precision LU keeps its working matrix as two float32 planes (real,
// imaginary), column-major.  A complex update C -= A B is one real GEMM in the
// "4M" embedding
//     [Cr | Ci] -= [Ar | Ai] * [[Br, Bi], [-Bi, Br]]
// with K' = 2k.  The LU panel kernels write the two operands already packed,
// K-major (K' contiguous per row / per output column):
//   Aop[b][row][K']   row i: [Re A(i, 0..k), Im A(i, 0..k)]
//   Bop[b][r][K']     per group of 128 complex output columns j0..j0+127, rows
//                     2*j0 + t   (t < 128): [ Re B(:, j0+t); -Im B(:, j0+t)]
//                     2*j0 + 128 + t     : [ Im B(:, j0+t);  Re B(:, j0+t)]
// A CTA owns a 128 x 128 complex tile of C (accumulator 128 lanes x 256 fp32
// columns: real parts then imaginary parts).  Warp 0 streams operand slices
// with TMA (128-byte swizzle) through a 2-stage shared-memory ring (two CTAs
// per SM, so that one CTA's epilogue overlaps the other's MMAs), one thread
// of warp 1 issues tcgen05.mma (M=128, N=256, K=8 per instruction), warps 2-9
// read the accumulator back with tcgen05.ld and apply C -= acc in place, the
// loads of C running ahead of the accumulator reads: two warps per 32-lane
// quarter of the accumulator, one for the real plane and one for the imaginary
// plane, so that twice as many loads of C are in flight (the update is bound
// by the read and write of C).
// Every mbarrier wait is bounded; on timeout the kernel records an error and
// still drains its own copies before freeing tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include "common.cuh"

namespace bem {
namespace {

constexpr int kTM = 128;            // tile rows
constexpr int kTNc = 128;           // tile complex columns
constexpr int kTN = 2 * kTNc;       // accumulator columns (MMA N)
constexpr int kKC = 32;             // K' values per stage (128 bytes of fp32)
constexpr int kStages = 2;
constexpr int kABytes = kTM * kKC * 4;   // 16 KiB
constexpr int kBBytes = kTN * kKC * 4;   // 32 KiB
constexpr int kStageBytes = kABytes + kBBytes;
constexpr int kTmemCols = 256;
constexpr long long kWaitLimit = 1ll << 20;  // try_wait polls; ends a stuck wait within seconds

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and records an error) when the limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  long long it = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++it > kWaitLimit) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms of
// 1024 bytes (stride byte offset 1024), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc_k_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1 << 46;            // version
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = 256.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct UpdateArgs {
  int a_row0;        // first operand row of the trailing block (Aop)
  int b_row0;        // first operand row of the trailing block (Bop), = 2 * first complex column
  int c_row0;        // first row of the trailing block in C
  int c_col0;        // first complex column of the trailing block in C
  int nk;            // K' / kKC
  int nk0;           // chunks read from the first operand pair; the rest from the second
  float* Cr;
  float* Ci;
  int64_t ldc;
  int64_t c_stride;  // elements between matrices
  int* err;
  int store;         // 0: C -= A B;  1: C = A B (C is not read)
};

constexpr int kThreads = 320;  // producer warp, MMA warp, 8 epilogue warps

__global__ void __launch_bounds__(kThreads, 2) cgemm_tf32_update_kernel(const __grid_constant__ CUtensorMap mapA,
                                                                   const __grid_constant__ CUtensorMap mapB,
                                                                   const __grid_constant__ CUtensorMap mapA1,
                                                                   const __grid_constant__ CUtensorMap mapB1,
                                                                   UpdateArgs p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment of the operand ring (128-byte swizzle atoms)
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char* ringA = smem;
  unsigned char* ringB = smem + kStages * kABytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accf = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accf + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tm = blockIdx.x, tn = blockIdx.y, b = blockIdx.z;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accf, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // producer
      bool ok = true;
      int issued = 0;
      for (int kc = 0; kc < p.nk && ok; ++kc) {
        const int s = kc % kStages;
        if (kc >= kStages) ok = mbar_wait(&empty[s], ((kc / kStages) - 1) & 1, p.err);
        if (!ok) break;
        mbar_expect_tx(&full[s], kStageBytes);
        // K' chunks [0, nk0) from the first operand pair, the rest from the second
        const bool first = kc < p.nk0;
        const int kx = (first ? kc : kc - p.nk0) * kKC;
        tma_load_3d(ringA + s * kABytes, first ? &mapA : &mapA1, kx, p.a_row0 + tm * kTM, b, &full[s]);
        tma_load_3d(ringB + s * kBBytes, first ? &mapB : &mapB1, kx, p.b_row0 + tn * kTN, b, &full[s]);
        issued = kc + 1;
      }
      // drain: every issued copy must land before the CTA may exit
      for (int kc = (issued > kStages ? issued - kStages : 0); kc < issued; ++kc)
        mbar_wait(&full[kc % kStages], (kc / kStages) & 1, p.err);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      bool ok = true;
      for (int kc = 0; kc < p.nk && ok; ++kc) {
        const int s = kc % kStages;
        ok = mbar_wait(&full[s], (kc / kStages) & 1, p.err);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t a0 = smem_u32(ringA + s * kABytes), b0 = smem_u32(ringB + s * kBBytes);
#pragma unroll
        for (int kk = 0; kk < kKC / 8; ++kk) {
          // K = 8 tf32 = 32 bytes per instruction inside the 128-byte swizzle atom
          mma_tf32(tmem, smem_desc_k_sw128(a0 + kk * 32), smem_desc_k_sw128(b0 + kk * 32), (kc | kk) != 0);
        }
        mma_commit(&empty[s]);
      }
      mma_commit(accf);
    }
  } else {
    // epilogue warps 2..9: TMEM lanes 32*(warp % 4) .. +31; warps 2-5 take the
    // real plane (accumulator columns 0..127), warps 6-9 the imaginary plane.
    // Each reads its plane in 8 chunks of 16 columns through a register double
    // buffer: the first chunk is loaded while the MMAs run, chunk i+1 while
    // chunk i is applied.
    constexpr int kCW = 16;                // columns per chunk
    constexpr int kPlaneChunks = kTNc / kCW;
    const int q = warp & 3;
    const int first = ((warp - 2) >> 2) * kPlaneChunks, last = first + kPlaneChunks;
    const int row = p.c_row0 + tm * kTM + 32 * q + lane;
    float* Cr = p.Cr + (size_t)b * p.c_stride + row;
    float* Ci = p.Ci + (size_t)b * p.c_stride + row;
    const int col0 = p.c_col0 + tn * kTNc;
    const int64_t ldc = p.ldc;
    auto at = [&](int chunk) -> float* {
      return (chunk < kPlaneChunks ? Cr : Ci) + (size_t)(col0 + (chunk % kPlaneChunks) * kCW) * ldc;
    };
    const bool rd = p.store == 0;
    float cb0[kCW], cb1[kCW];
#pragma unroll
    for (int j = 0; j < kCW; ++j) cb0[j] = cb1[j] = 0.0f;
    if (rd) {
      const float* src = at(first);
#pragma unroll
      for (int j = 0; j < kCW; ++j) cb0[j] = __ldcs(src + j * ldc);
    }
    const bool ok = __all_sync(0xffffffffu, mbar_wait(accf, 0, p.err));
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    __syncwarp();
    if (ok) {
      const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16);
#pragma unroll 1
      for (int chunk = first; chunk < last; chunk += 2) {
        if (rd) {
          const float* src = at(chunk + 1);
#pragma unroll
          for (int j = 0; j < kCW; ++j) cb1[j] = __ldcs(src + j * ldc);
        }
        {
          float v[kCW];
          tmem_ld16(tbase + (uint32_t)(chunk * kCW), v);
          float* dst = at(chunk);
#pragma unroll
          for (int j = 0; j < kCW; ++j) __stcs(dst + j * ldc, rd ? cb0[j] - v[j] : v[j]);
        }
        if (rd && chunk + 2 < last) {
          const float* src = at(chunk + 2);
#pragma unroll
          for (int j = 0; j < kCW; ++j) cb0[j] = __ldcs(src + j * ldc);
        }
        {
          float v[kCW];
          tmem_ld16(tbase + (uint32_t)((chunk + 1) * kCW), v);
          float* dst = at(chunk + 1);
#pragma unroll
          for (int j = 0; j < kCW; ++j) __stcs(dst + j * ldc, rd ? cb1[j] - v[j] : v[j]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// cuTensorMapEncodeTiled resolved through the runtime, so that the library
// loads on hosts without a GPU driver (no link-time libcuda dependency).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor map of a packed operand: float32 [batch][rows][kp], box {32, box_rows, 1}.
int make_operand_map(CUtensorMap* map, const float* base, int kp, int64_t rows, int batch, int box_rows) {
  auto encode = encode_fn();
  if (!encode) return set_error(BEM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[3] = {(cuuint64_t)kp, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)kp * 4, (cuuint64_t)kp * 4 * (cuuint64_t)rows};
  cuuint32_t box[3] = {(cuuint32_t)kKC, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims,
                                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(BEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return BEM_OK;
}

bool g_tc_configured = false;

}  // namespace

// Host entry shared with the LU: C (trailing block m x n complex, both multiples
// of 128) -= A' B' for `batch` matrices.
int cgemm_tf32_update(const float* Aop, int64_t a_rows, int a_row0, const float* Bop, int64_t b_rows, int b_row0,
                      int kp, float* Cr, float* Ci, int64_t ldc, int64_t c_stride, int c_row0, int c_col0, int m,
                      int n, int batch, int* err, cudaStream_t stream, int store, const float* Aop1,
                      const float* Bop1) {
  if (m <= 0 || n <= 0) return BEM_OK;
  if (m % kTM || n % kTNc || kp % kKC || (a_row0 % 8) || (b_row0 % 8))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "cgemm_tf32_update: sizes must be multiples of 128 (K' of 32)");
  if ((Aop1 == nullptr) != (Bop1 == nullptr))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "cgemm_tf32_update: second operand pair incomplete");
  CUtensorMap mapA, mapB, mapA1, mapB1;
  int st = make_operand_map(&mapA, Aop, kp, a_rows, batch, kTM);
  if (st) return st;
  st = make_operand_map(&mapB, Bop, kp, b_rows, batch, kTN);
  if (st) return st;
  // second pair (same shapes, the next K' block): C -= A B - A1 B1 in one pass over C
  st = make_operand_map(&mapA1, Aop1 ? Aop1 : Aop, kp, a_rows, batch, kTM);
  if (st) return st;
  st = make_operand_map(&mapB1, Bop1 ? Bop1 : Bop, kp, b_rows, batch, kTN);
  if (st) return st;
  const int smem = kStages * kStageBytes + 1024 + 256;
  if (!g_tc_configured) {
    BEM_CUDA_CHECK(cudaFuncSetAttribute(cgemm_tf32_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    g_tc_configured = true;
  }
  const int nk0 = kp / kKC;
  UpdateArgs p{a_row0, b_row0, c_row0, c_col0, Aop1 ? 2 * nk0 : nk0, nk0, Cr, Ci, ldc, c_stride, err, store};
  dim3 grid(m / kTM, n / kTNc, batch);
  {
    TimedLaunch tl(kKCgemmTf32, stream);
    cgemm_tf32_update_kernel<<<grid, kThreads, smem, stream>>>(mapA, mapB, mapA1, mapB1, p);
  }
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

}  // namespace bem

extern "C" int bem_cgemm_tf32_update(const float* Aop_dev, int64_t a_rows, int a_row0, const float* Bop_dev,
                                     int64_t b_rows, int b_row0, int kp, float* Cr_dev, float* Ci_dev, int64_t ldc,
                                     int64_t c_stride, int c_row0, int c_col0, int m, int n, int batch, int* err_dev,
                                     void* stream) {
  if (!Aop_dev || !Bop_dev || !Cr_dev || !Ci_dev || !err_dev || batch <= 0 || ldc < c_row0 + m || kp <= 0)
    return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bem_cgemm_tf32_update: bad arguments");
  if ((int64_t)a_row0 + m > a_rows || (int64_t)b_row0 + 2 * (int64_t)n > b_rows)
    return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bem_cgemm_tf32_update: operand rows out of range");
  if ((reinterpret_cast<uintptr_t>(Aop_dev) | reinterpret_cast<uintptr_t>(Bop_dev)) & 15)
    return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bem_cgemm_tf32_update: operands must be 16-byte aligned");
  return bem::cgemm_tf32_update(Aop_dev, a_rows, a_row0, Bop_dev, b_rows, b_row0, kp, Cr_dev, Ci_dev, ldc, c_stride,
                                c_row0, c_col0, m, n, batch, err_dev, (cudaStream_t)stream, 0, nullptr, nullptr);
}
