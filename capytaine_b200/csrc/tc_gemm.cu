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
#include <algorithm>
#include "common.cuh"

namespace bem {
namespace {

constexpr int kTM = 128;            // tile rows
constexpr int kTNc = 128;           // tile complex columns
constexpr int kTN = 2 * kTNc;       // accumulator columns (MMA N)
constexpr int kKC = 32;             // K' values per stage (128 bytes of fp32)
constexpr int kStages = 4;
constexpr int kABytes = kTM * kKC * 4;   // 16 KiB
constexpr int kBBytes = kTN * kKC * 4;   // 32 KiB
constexpr int kStageBytes = kABytes + kBBytes;
constexpr long long kWaitLimit = 1ll << 22;  // default polls of a bounded mbarrier wait (~ a second)
constexpr int kMaxGroup = 64;  // matrices of one grouped launch

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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
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
  int tiles_m;       // tile grid: tiles_m x tiles_n x batch, tm fastest
  int tiles_n;
  int ntiles;
  int waves;             // CTA groups, each over its own range of consecutive tiles
  int group_width;       // CTAs per group (at most the SM count)
  long long wait_limit;  // polls of a bounded mbarrier wait
  // Grouped launch (ngroup > 0): matrix b has gtm[b] x gtn[b] tiles of its own,
  // tiles gstart[b] .. gstart[b+1]-1 (matrices of different active sizes)
  int ngroup;
  int batch0;  // matrix index of local matrix 0 (operand batch coordinate, C offset)
  // Packed copy of the result for the next block step's products (kPack*):
  // the operand layouts the LU's update reads, written by the epilogue
  float* pack;
  int64_t pack_stride;  // floats between matrices
  int pack_mode;
  // L-shaped launch: only the first tile row and the first tile column of the
  // m x n block, without the corner tile (R = tiles_m - 1 of each; grouped:
  // R of matrix b in gtm[b])
  int lshape;
  int gstart[kMaxGroup + 1];
  short gtm[kMaxGroup];
  short gtn[kMaxGroup];
};

// Matrix and tile coordinates of tile t of the launch.
__device__ __forceinline__ void decode_tile(const UpdateArgs& p, int t, int& b, int& tm, int& tn) {
  if (p.lshape) {
    int R, r;
    if (p.ngroup > 0) {
      b = 0;
      while (b + 1 < p.ngroup && p.gstart[b + 1] <= t) ++b;
      R = p.gtm[b];
      r = t - p.gstart[b];
    } else {
      R = p.tiles_m - 1;
      b = t / (2 * R);
      r = t - b * 2 * R;
    }
    if (r < R) {
      tm = 0;
      tn = r + 1;
    } else {
      tm = r - R + 1;
      tn = 0;
    }
    return;
  }
  if (p.ngroup > 0) {
    b = 0;
    while (b + 1 < p.ngroup && p.gstart[b + 1] <= t) ++b;
    const int r = t - p.gstart[b];
    tn = r / p.gtm[b];
    tm = r - tn * p.gtm[b];
    return;
  }
  const int per_matrix = p.tiles_m * p.tiles_n;
  b = t / per_matrix;
  const int r = t - b * per_matrix;
  tn = r / p.tiles_m;
  tm = r - tn * p.tiles_m;
}

constexpr int kEpiWarps = 16;                  // 4 lane quarters x 4 groups of 64 accumulator columns
constexpr int kThreads = 32 * (2 + kEpiWarps);  // producer warp, MMA warp, epilogue warps
constexpr int kAccCols = kTN;                  // TMEM columns of one accumulator
constexpr int kTmemAlloc = 2 * kAccCols;       // two accumulators: all 512 columns of the SM

// Bounded wait with the limit of the launch.
__device__ __forceinline__ bool mbar_wait_n(uint64_t* bar, uint32_t parity, int* err, long long limit) {
  long long it = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++it > limit) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// Packed copy of 16 result values of one thread (row layout [Re | Im], 256
// floats per row), rounded to TF32 (it is an operand of later products): off
// is the offset from the thread's pack pointer.
__device__ __forceinline__ void pack_chunk(float* pk, int off, const float (&v)[16]) {
  float4* d = reinterpret_cast<float4*>(pk + off);
#pragma unroll
  for (int j = 0; j < 4; ++j)
    d[j] = make_float4(tf32_rn(v[4 * j]), tf32_rn(v[4 * j + 1]), tf32_rn(v[4 * j + 2]), tf32_rn(v[4 * j + 3]));
}

// Trailing update with double-buffered accumulators: a CTA (one per SM: 197 KB
// of shared memory, all 512 tensor-memory columns) takes a run of 128 x 128
// complex tiles (an even share of its group's tile range), spaced so that the
// CTAs of a group work on consecutive tiles at any time (their operands stay
// in L2), and alternates between two accumulators in tensor memory, so that
// the epilogue of tile i (read C, subtract, write C) overlaps the MMAs of tile
// i+1.  CTAs retire after their run, so kernels of other streams (the
// lookahead of the block LU) get SMs within one run.  Barriers: full/empty per
// operand stage (TMA -> MMA -> TMA),
// acc_full per accumulator (MMA commit -> epilogue), acc_empty per
// accumulator (one arrival per epilogue warp -> MMA).
__global__ void __launch_bounds__(kThreads, 1) cgemm_tf32_update_kernel(const __grid_constant__ CUtensorMap mapA,
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
  uint64_t* acc_full = empty + kStages;  // [2]
  uint64_t* acc_empty = acc_full + 2;    // [2]
  uint64_t* mma_done = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long limit = p.wait_limit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], kEpiWarps);
    }
    mbar_init(mma_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemAlloc)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  // This CTA's tiles: `waves` groups of group_width CTAs (one CTA per SM);
  // group g covers the tiles [g N / G, (g+1) N / G) and its CTA l takes the
  // tiles start + l + j W, so the CTAs of a group work on W consecutive tiles
  // at a time (tm fastest: they share the operands in L2), every CTA of a
  // group has the same number of tiles to within one, and each retires after
  // its share (the next group takes its SM).
  const int Wg = p.group_width;
  const int grp = blockIdx.x / Wg, l = blockIdx.x - grp * Wg;
  const int t_first = (int)((long long)grp * p.ntiles / p.waves) + l;
  const int t_end = (int)((long long)(grp + 1) * p.ntiles / p.waves);

  if (warp == 0) {
    if (lane == 0) {
      // producer: operand slices of every tile of this CTA through the ring
      bool ok = true;
      long long g = 0;  // stage uses so far
      for (int t = t_first; t < t_end && ok; t += Wg) {
        int b, tm, tn;
        decode_tile(p, t, b, tm, tn);
        b += p.batch0;
        for (int kc = 0; kc < p.nk; ++kc, ++g) {
          const int s = (int)(g % kStages);
          const uint32_t use = (uint32_t)(g / kStages);
          if (g >= kStages && !(ok = mbar_wait_n(&empty[s], (use - 1) & 1, p.err, limit))) break;
          mbar_expect_tx(&full[s], kStageBytes);
          // K' chunks [0, nk0) from the first operand pair, the rest from the second
          const bool first = kc < p.nk0;
          const int kx = (first ? kc : kc - p.nk0) * kKC;
          tma_load_3d(ringA + s * kABytes, first ? &mapA : &mapA1, kx, p.a_row0 + tm * kTM, b, &full[s]);
          tma_load_3d(ringB + s * kBBytes, first ? &mapB : &mapB1, kx, p.b_row0 + tn * kTN, b, &full[s]);
        }
      }
      // drain: every issued copy must land before the CTA may exit
      for (long long q = (g > kStages ? g - kStages : 0); q < g; ++q)
        mbar_wait_n(&full[q % kStages], (uint32_t)(q / kStages) & 1, p.err, limit);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      bool ok = true;
      long long g = 0;
      int i = 0;  // tiles of this CTA so far
      for (int t = t_first; t < t_end && ok; t += Wg, ++i) {
        const int acc = i & 1;
        const uint32_t use = (uint32_t)(i >> 1);
        // the epilogue must have drained this accumulator's previous tile
        if (i >= 2 && !(ok = mbar_wait_n(&acc_empty[acc], (use - 1) & 1, p.err, limit))) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t tacc = tmem + (uint32_t)(acc * kAccCols);
        for (int kc = 0; kc < p.nk; ++kc, ++g) {
          const int s = (int)(g % kStages);
          if (!(ok = mbar_wait_n(&full[s], (uint32_t)(g / kStages) & 1, p.err, limit))) break;
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t a0 = smem_u32(ringA + s * kABytes), b0 = smem_u32(ringB + s * kBBytes);
#pragma unroll
          for (int kk = 0; kk < kKC / 8; ++kk) {
            // K = 8 tf32 = 32 bytes per instruction inside the 128-byte swizzle atom
            mma_tf32(tacc, smem_desc_k_sw128(a0 + kk * 32), smem_desc_k_sw128(b0 + kk * 32), (kc | kk) != 0);
          }
          mma_commit(&empty[s]);
        }
        if (!ok) break;
        mma_commit(&acc_full[acc]);
      }
      // every MMA issued by this thread has completed before tensor memory is freed
      mma_commit(mma_done);
      mbar_wait_n(mma_done, 0, p.err, limit);
    }
  } else {
    // epilogue warp: TMEM lanes 32 q .. 32 q + 31 (q = warp % 4, the quarter a
    // warp may access), accumulator columns 64 cg .. 64 cg + 63 (cg 0, 1: real
    // plane; 2, 3: imaginary plane), in 4 chunks of 16 columns through a
    // register double buffer of C.
    constexpr int kCW = 16;
    constexpr int kChunks = 64 / kCW;
    const int q = warp & 3, cg = (warp - 2) >> 2;
    const int plane = cg >> 1, cbase = (cg & 1) * 64;
    const bool rd = p.store == 0;
    const int64_t ldc = p.ldc;
    bool ok = true;
    int i = 0;
    for (int t = t_first; t < t_end && ok; t += Wg, ++i) {
      int b, tm, tn;
      decode_tile(p, t, b, tm, tn);
      b += p.batch0;
      const int acc = i & 1;
      const int row = p.c_row0 + tm * kTM + 32 * q + lane;
      float* C = (plane ? p.Ci : p.Cr) + (size_t)b * p.c_stride + row +
                 (size_t)(p.c_col0 + tn * kTNc + cbase) * ldc;
      float cb0[kCW], cb1[kCW];
#pragma unroll
      for (int j = 0; j < kCW; ++j) cb0[j] = cb1[j] = 0.0f;
      if (rd) {
#pragma unroll
        for (int j = 0; j < kCW; ++j) cb0[j] = __ldcs(C + (size_t)j * ldc);
      }
      ok = __all_sync(0xffffffffu, mbar_wait_n(&acc_full[acc], (uint32_t)(i >> 1) & 1, p.err, limit));
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (!ok) break;
      const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * kAccCols + plane * kTNc + cbase);
      // packed copy: this thread's row of the tile
      float* pk = p.pack_mode == kPackRows
                      ? p.pack + (size_t)b * p.pack_stride + (size_t)row * kTN + plane * kTNc + cbase
                      : nullptr;
#pragma unroll
      for (int chunk = 0; chunk < kChunks; chunk += 2) {
        if (rd) {
#pragma unroll
          for (int j = 0; j < kCW; ++j) cb1[j] = __ldcs(C + (size_t)((chunk + 1) * kCW + j) * ldc);
        }
        {
          float v[kCW];
          tmem_ld16(tbase + (uint32_t)(chunk * kCW), v);
#pragma unroll
          for (int j = 0; j < kCW; ++j) {
            v[j] = rd ? cb0[j] - v[j] : v[j];
            __stcs(C + (size_t)(chunk * kCW + j) * ldc, v[j]);
          }
          if (pk) pack_chunk(pk, chunk * kCW, v);
        }
        if (rd && chunk + 2 < kChunks) {
#pragma unroll
          for (int j = 0; j < kCW; ++j) cb0[j] = __ldcs(C + (size_t)((chunk + 2) * kCW + j) * ldc);
        }
        {
          float v[kCW];
          tmem_ld16(tbase + (uint32_t)((chunk + 1) * kCW), v);
#pragma unroll
          for (int j = 0; j < kCW; ++j) {
            v[j] = rd ? cb1[j] - v[j] : v[j];
            __stcs(C + (size_t)((chunk + 1) * kCW + j) * ldc, v[j]);
          }
          if (pk) pack_chunk(pk, (chunk + 1) * kCW, v);
        }
      }
      // this warp's reads of the accumulator are complete: release it
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[acc]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemAlloc) : "memory");
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
int g_num_sms[64] = {0};

int num_sms(int* out) {
  int dev = 0;
  BEM_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BEM_ERR_UNSUPPORTED, "device index out of range");
  if (!g_num_sms[dev]) BEM_CUDA_CHECK(cudaDeviceGetAttribute(&g_num_sms[dev], cudaDevAttrMultiProcessorCount, dev));
  *out = g_num_sms[dev];
  return BEM_OK;
}

}  // namespace

// Host entry shared with the LU: C (trailing block m x n complex, both multiples
// of 128) -= A' B' for `batch` matrices.  run > 0: tiles per CTA; 0: chosen
// from the tile count (up to 32 while there are at least two runs per SM).
int cgemm_tf32_update(const float* Aop, int64_t a_rows, int a_row0, const float* Bop, int64_t b_rows, int b_row0,
                      int kp, float* Cr, float* Ci, int64_t ldc, int64_t c_stride, int c_row0, int c_col0, int m,
                      int n, int batch, int* err, cudaStream_t stream, int store, const float* Aop1,
                      const float* Bop1, int run, long long wait_limit, const int* limit_host, float* pack,
                      int pack_mode, int64_t pack_stride, bool lshape, int reserve_sms) {
  if (m <= 0 || n <= 0) return BEM_OK;
  if (lshape && (m != n || m <= kTM || pack_mode != kPackNone))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "cgemm_tf32_update: an L-shaped update needs a square block of "
                                               "more than one tile and no packed copy");
  if (pack_mode != kPackNone &&
      (pack_mode != kPackRows || !pack || n != kTNc || (reinterpret_cast<uintptr_t>(pack) & 15)))
    return set_error(BEM_ERR_INVALID_ARGUMENT,
                     "cgemm_tf32_update: a packed copy needs one tile column and a 16-byte aligned destination");
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
  int sms = 0;
  if ((st = num_sms(&sms))) return st;
  const int nk0 = kp / kKC;
  const int tiles_m = m / kTM, tiles_n = n / kTNc;
  UpdateArgs p{};
  p.a_row0 = a_row0;
  p.b_row0 = b_row0;
  p.c_row0 = c_row0;
  p.c_col0 = c_col0;
  p.nk = Aop1 ? 2 * nk0 : nk0;
  p.nk0 = nk0;
  p.Cr = Cr;
  p.Ci = Ci;
  p.ldc = ldc;
  p.c_stride = c_stride;
  p.err = err;
  p.store = store;
  p.tiles_m = tiles_m;
  p.tiles_n = tiles_n;
  p.wait_limit = wait_limit > 0 ? wait_limit : kWaitLimit;
  p.pack = pack;
  p.pack_stride = pack_stride;
  p.pack_mode = pack_mode;
  p.lshape = lshape ? 1 : 0;
  int launches = 0;
  // Grouped: matrix b covers only rows and columns below limit_host[b] (its
  // active size), launches of at most kMaxGroup matrices
  for (int b0 = 0; b0 < batch; b0 += limit_host ? kMaxGroup : batch) {
    const int nb = limit_host ? std::min(kMaxGroup, batch - b0) : batch;
    long long ntiles = lshape ? 2ll * (tiles_m - 1) * nb : (long long)tiles_m * tiles_n * nb;
    if (limit_host) {
      p.ngroup = nb;
      ntiles = 0;
      for (int i = 0; i < nb; ++i) {
        const int lim = limit_host[b0 + i];
        const int mb = std::max(0, std::min(m, lim - c_row0)) / kTM;
        const int nbc = std::max(0, std::min(n, lim - c_col0)) / kTNc;
        p.gstart[i] = (int)ntiles;
        if (lshape) {  // R tiles in the row and R in the column beyond the corner
          const int R = std::max(0, mb - 1);
          p.gtm[i] = (short)R;
          p.gtn[i] = 0;
          ntiles += 2ll * R;
          continue;
        }
        p.gtm[i] = (short)std::max(mb, 1);  // never divides by zero; no tile when gtn is 0
        p.gtn[i] = (short)(mb > 0 ? nbc : 0);
        ntiles += (long long)(mb > 0 ? mb : 0) * (mb > 0 ? nbc : 0);
      }
      p.gstart[nb] = (int)ntiles;
    }
    if (ntiles > (1ll << 30)) return set_error(BEM_ERR_INVALID_ARGUMENT, "cgemm_tf32_update: too many tiles");
    if (ntiles == 0) continue;
    p.ntiles = (int)ntiles;
    // groups of up to one CTA per SM, each CTA with about `per` tiles (run, or
    // up to 32 for the big updates so that other streams get SMs within a run);
    // reserve_sms SMs held by a kernel running beside this one are left out of
    // the width, so that a group never waits for them with its share of tiles
    const long long per = run > 0 ? run : 32;
    const long long avail = std::max(1, sms - std::min(std::max(0, reserve_sms), sms / 2));
    const long long waves = (ntiles + avail * per - 1) / (avail * per);
    const long long width = std::min<long long>(avail, (ntiles + waves * (run > 0 ? run : 1) - 1) /
                                                           (waves * (run > 0 ? run : 1)));
    const long long ctas = waves * width;
    UpdateArgs q = p;
    q.waves = (int)waves;
    q.group_width = (int)width;
    q.batch0 = b0;  // the matrices of this launch: b0 .. b0 + nb - 1
    {
      TimedLaunch tl(kKCgemmTf32, stream);
      cgemm_tf32_update_kernel<<<(unsigned)ctas, kThreads, smem, stream>>>(mapA, mapB, mapA1, mapB1, q);
    }
    ++launches;
  }
  count_launches(launches);
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
                                c_row0, c_col0, m, n, batch, err_dev, (cudaStream_t)stream, 0, nullptr, nullptr, 0, 0,
                                nullptr, nullptr, bem::kPackNone, 0, false, 0);
}
