// tc_dft.cuh -- 1024-point complex DFT of lines on the fifth-generation
// tensor cores (tcgen05.mma), with split-BF16 operands accumulated in FP32.
//
// This is the mixed-precision form of the radix-32 FFT passes of
// fft_core.cuh, i.e. of the reference's FFTW 1-D transforms (planned in
// PSDNS/epfftw.f; executed at PSDNS/itransform_vel.f:88,
// PSDNS/kxcomm1_clean.f:118, PSDNS/transform.f:134, PSDNS/xkcomm2.f:229,
// PSDNS/xkcomm1.f:97).
//
// Algorithm (four steps, 1024 = 32 x 32).  With n = 32 n1 + n2 and
// k = k1 + 32 k2,
//     X[k1 + 32 k2] = sum_n2 W32^(n2 k2) W1024^(n2 k1) sum_n1 W32^(n1 k1) x[32 n1 + n2],
// W_m = exp(-2 pi i / m).  Both DFT-32 sums are real matrix products: a
// complex row (re | im, 64 values) times the 64 x 64 real form of the DFT-32
// matrix gives the transformed row (re | im).  Four lines form an M = 128
// tile (row 32 q + n2 is line q's n2; N = 64, K = 64).  Every operand is
// split into two BF16 numbers, v = v_hi + v_lo, and the three products
// x_hi F_hi + x_hi F_lo + x_lo F_hi accumulate in FP32 in tensor memory; the
// dropped x_lo F_lo term and the residuals of the splits are of relative
// size 2^-16 to 2^-17 per operand.  The twiddle W1024^(n2 k1) between the
// two products is applied in FP32 to the FP32 accumulator.
//
// Operand layouts (shared memory, no swizzle, 8 x 16-byte core matrices):
//   A (data, MN-major): element (m, k) at (k/8)*2048 + (m/8)*128 + (k%8)*16 + (m%8)*2
//                       bytes: leading (K) byte offset 2048, stride (M) 128;
//                       hi part at +0, lo part at +16384 (one tile: 32 KB)
//   B (DFT-32, K-major): element (n, k) at (n/8)*1024 + (k/8)*128 + (n%8)*16 + (k%8)*2
//                       bytes: leading (K) byte offset 128, stride (N) 1024;
//                       hi at +0, lo at +8192 (16 KB, built on the host)
// The accumulator of tile t is TMEM lanes 0..127 x columns 64 t .. 64 t + 63:
// lane m = row m, column c = output c (re of k for c < 32, im of k - 32).
// Warp w of the block owns line w (the stage kernels run one warp per line
// at n = 1024), so its rows are TMEM lanes 32 (w % 4) .. + 31 of tile w / 4,
// exactly the lane quarter that warp may read.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_core.cuh"

namespace psdns {
namespace tc {

constexpr int kTileBytes = 32768;   // A hi + A lo of one tile (4 lines)
constexpr int kBBytes = 16384;      // B hi + B lo
constexpr int kLoOff = 16384;       // lo part of A
constexpr int kBLoOff = 8192;       // lo part of B
// bounded waits: a thread gives up on an MMA completion after this many
// nanoseconds of the global timer and flags an error (an MMA tile takes
// well under a microsecond)
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

// instruction descriptor of tcgen05.mma kind::f16: D FP32 (bits 4-5 = 1),
// A and B BF16 (bits 7-9 and 10-12 = 1), A major (bit 15), B K-major
// (bit 16 = 0), N >> 3 (bits 17-22), M >> 4 (bits 24-28)
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (all >> 4), descriptor version 1 at bit 46
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// wait for the phase with the given parity to complete; false if the time
// bound ran out (each try_wait suspends for at most 1 microsecond)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const uint32_t a = smem_u32(bar);
  const unsigned long long t0 = global_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(1000u)
        : "memory");
    if (ok) return true;
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
}

// D[tmem] (+)= A B^T, M x N x 16, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on the mbarrier once every tcgen05 operation issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// whole warp: allocate NCOLS tensor-memory columns, address written to *slot
template <int NCOLS>
__device__ __forceinline__ void tmem_alloc(uint32_t* slot) {
  static_assert(NCOLS >= 32 && NCOLS <= 512 && (NCOLS & (NCOLS - 1)) == 0, "TMEM columns: power of two >= 32");
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(NCOLS)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
template <int NCOLS>
__device__ __forceinline__ void tmem_free(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(NCOLS) : "memory");
}

// 32 consecutive columns of this thread's lane (lane quarter of the warp)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// v = hi + lo, both round-to-nearest BF16; returned as raw 16-bit patterns
__device__ __forceinline__ void split_bf16(float v, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat16_raw h = __nv_bfloat16_raw(__float2bfloat16_rn(v));
  const float r = v - __bfloat162float(__nv_bfloat16(h));
  const __nv_bfloat16_raw l = __nv_bfloat16_raw(__float2bfloat16_rn(r));
  hi = h.x;
  lo = l.x;
}

// 8 floats -> 16-byte rows of the hi and lo operands
__device__ __forceinline__ void split8(const float* v, uint4& hi, uint4& lo) {
  uint32_t h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; i++) split_bf16(v[i], h[i], l[i]);
  hi = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
  lo = make_uint4(l[0] | (l[1] << 16), l[2] | (l[3] << 16), l[4] | (l[5] << 16), l[6] | (l[7] << 16));
}

// byte offset of element (m, k) in the MN-major A layout, for 8 consecutive m
__host__ __device__ __forceinline__ constexpr int a_off(int m, int k) {
  return (k >> 3) * 2048 + (m >> 3) * 128 + (k & 7) * 16 + (m & 7) * 2;
}
// byte offset of element (n, k) in the K-major B layout
__host__ __device__ __forceinline__ constexpr int b_off(int n, int k) {
  return (n >> 3) * 1024 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
}

// state of the tensor-core transform of one thread block
struct Work {
  uint32_t tmem;     // TMEM base address (lane 0, first column)
  uint32_t b;        // shared-memory address of the B operands (hi, then lo)
  uint64_t* bar;     // completion barrier of the MMAs
  unsigned phase;    // parity of the next completion
  unsigned* err;     // global error word (bit 0: an MMA wait ran out)
  const float2* tw;  // W1024^(n2 k1) as [k1][n2] (global memory, cached)
};

// Block set-up: copy the B operands into shared memory, initialise the
// barrier, allocate NCOLS TMEM columns (warp 0).  Called by every thread.
template <int NCOLS>
__device__ __forceinline__ void setup(Work& w, unsigned char* bsmem, uint64_t* bar, uint32_t* tslot,
                                      const uint4* __restrict__ btab, const float2* __restrict__ tw,
                                      unsigned* err) {
  for (int i = threadIdx.x; i < kBBytes / 16; i += blockDim.x) {
    const uint32_t s = smem_u32(bsmem + 16 * i);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(btab + i) : "memory");
  }
  if (threadIdx.x == 0) mbar_init(bar, 1);
  if (threadIdx.x < 32) tmem_alloc<NCOLS>(tslot);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  w.tmem = *tslot;
  w.b = smem_u32(bsmem);
  w.bar = bar;
  w.phase = 0;
  w.err = err;
  w.tw = tw;
}

// Block tear-down: free the TMEM columns (warp 0).  Called by every thread.
template <int NCOLS>
__device__ __forceinline__ void teardown(const Work& w) {
  fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after();
    tmem_free<NCOLS>(w.tmem);
  }
}

// one thread: the 12 MMAs (3 split products x 4 K-steps) of every tile
__device__ __forceinline__ void issue_tiles(const Work& w, uint32_t tile0, uint32_t tile_stride, int ntiles) {
  constexpr uint32_t idesc = idesc_bf16(128, 64, true);
  for (int t = 0; t < ntiles; t++) {
    const uint32_t a = tile0 + t * tile_stride;
    const uint32_t d = w.tmem + 64u * t;
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const uint32_t ap = a + (p == 2 ? kLoOff : 0);
      const uint32_t bp = w.b + (p == 1 ? kBLoOff : 0);
#pragma unroll
      for (int s = 0; s < 4; s++)
        mma_bf16(d, sdesc(ap + s * 4096, 2048, 128), sdesc(bp + s * 256, 128, 1024), idesc,
                 (p > 0 || s > 0) ? 1u : 0u);
    }
  }
}

// the MMAs of all tiles: operands written -> issue -> wait
__device__ __forceinline__ void run_mmas(Work& w, uint32_t tile0, uint32_t tile_stride, int ntiles) {
  fence_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_after();
    issue_tiles(w, tile0, tile_stride, ntiles);
    mma_commit(w.bar);
  }
  if (!mbar_wait(w.bar, w.phase) && (threadIdx.x & 31) == 0) atomicOr(w.err, 1u);
  w.phase ^= 1u;
  fence_after();
}

// Forward DFT (natural order in and out) of nlines <= THREADS/32 lines of
// 1024 complex FP32 values, warp l transforming line l.  The caller supplies
// the operands and takes the results through callbacks: s = lbegin(l), then
// load(s, i) returns element i of line l (i = 8 g + e for the thread's
// groups g = lane + 32 j); t = sbegin(l), then store(t, k, v) receives
// output k = lane + 32 k2.  tiles: shared memory for ceil(nlines/4) operand
// tiles of 32 KB, tstride bytes apart (16-byte aligned); every thread's
// loads complete before the first tile is written, so the tiles may overlay
// the input.  Called by every thread of the block; the stores are issued
// after the last block-wide barrier.
template <int THREADS, typename LBegin, typename Load, typename SBegin, typename Store>
__device__ __forceinline__ void fft1024(int nlines, Work& w, unsigned char* tiles, uint32_t tstride,
                                        LBegin lbegin, Load load, SBegin sbegin, Store store) {
  static_assert(THREADS % 32 == 0, "whole warps");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3;
  const int ntiles = (nlines + 3) >> 2;
  const bool in_tile = warp < 4 * ntiles;
  const bool act = warp < nlines;
  unsigned char* tile = tiles + (size_t)(warp >> 2) * tstride;
  const uint32_t tile0 = smem_u32(tiles);
  const uint32_t trow = w.tmem + ((uint32_t)(32 * q) << 16) + 64u * (warp >> 2);

  // stage 1 operand: thread holds groups g = lane + 32 j of 8 consecutive
  // elements 8 g .. 8 g + 7 (n1 = g / 4, n2 = 8 (g % 4) + e)
  float re[32], im[32];
  if (act) {
    const auto s = lbegin(warp);
    float2 v[32];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 8; e++) v[8 * j + e] = load(s, 8 * (lane + 32 * j) + e);
#pragma unroll
    for (int i = 0; i < 32; i++) {
      re[i] = v[i].x;
      im[i] = v[i].y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 32; i++) re[i] = im[i] = 0.f;
  }
  __syncthreads();   // every input is read before the tiles are written
  if (in_tile) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int g = lane + 32 * j, n1 = g >> 2, m = 32 * q + 8 * (g & 3);
      uint4 h, l;
      split8(re + 8 * j, h, l);
      *reinterpret_cast<uint4*>(tile + a_off(m, n1)) = h;
      *reinterpret_cast<uint4*>(tile + kLoOff + a_off(m, n1)) = l;
      split8(im + 8 * j, h, l);
      *reinterpret_cast<uint4*>(tile + a_off(m, 32 + n1)) = h;
      *reinterpret_cast<uint4*>(tile + kLoOff + a_off(m, 32 + n1)) = l;
    }
  }
  run_mmas(w, tile0, tstride, ntiles);

  // stage 1 result: lane n2, columns k1 (re) and 32 + k1 (im); twiddle
  if (in_tile) {
    tmem_ld32(trow, re);
    tmem_ld32(trow + 32, im);
#pragma unroll
    for (int k1 = 0; k1 < 32; k1++) {
      const float2 t = __ldg(w.tw + k1 * 32 + lane);
      const float a = re[k1], b = im[k1];
      re[k1] = a * t.x - b * t.y;
      im[k1] = a * t.y + b * t.x;
    }
  }
  fence_before();
  __syncthreads();   // stage-1 accumulators read; the tiles are free again
  // stage 2 operand: row 32 q + k1, K = n2 (re) / 32 + n2 (im), n2 = lane
  if (in_tile) {
#pragma unroll
    for (int kb = 0; kb < 4; kb++) {
      const int m = 32 * q + 8 * kb;
      uint4 h, l;
      split8(re + 8 * kb, h, l);
      *reinterpret_cast<uint4*>(tile + a_off(m, lane)) = h;
      *reinterpret_cast<uint4*>(tile + kLoOff + a_off(m, lane)) = l;
      split8(im + 8 * kb, h, l);
      *reinterpret_cast<uint4*>(tile + a_off(m, 32 + lane)) = h;
      *reinterpret_cast<uint4*>(tile + kLoOff + a_off(m, 32 + lane)) = l;
    }
  }
  run_mmas(w, tile0, tstride, ntiles);

  // stage 2 result: lane k1, columns k2 (re) and 32 + k2 (im) = X[k1 + 32 k2]
  if (in_tile) {
    tmem_ld32(trow, re);
    tmem_ld32(trow + 32, im);
  }
  fence_before();
  __syncthreads();   // the tiles are free
  if (act) {
    const auto t = sbegin(warp);
#pragma unroll
    for (int k2 = 0; k2 < 32; k2++) store(t, lane + 32 * k2, make_float2(re[k2], im[k2]));
  }
}

// fft1024 on lines held in shared memory, line l at buf + l ls, element i
// at pad32(i) (the layout of fft_lines), in place.  The operand tiles
// overlay lines 4t .. 4t + 3 (ls * 8 * 4 >= 32 KB bytes, 16-byte aligned):
// the storage of every line up to the next multiple of four is
// overwritten.  Ends with a barrier.
template <int THREADS>
__device__ __forceinline__ void fft1024_lines(float2* buf, int nlines, int ls, Work& w) {
  auto line = [&](int l) { return buf + (size_t)l * ls; };
  fft1024<THREADS>(
      nlines, w, reinterpret_cast<unsigned char*>(buf), (uint32_t)(4 * ls * sizeof(float2)), line,
      [](const float2* p, int i) { return p[pad32(i)]; }, line, [](float2* p, int k, float2 v) { p[pad32(k)] = v; });
  __syncthreads();
}

// Host: B operands (DFT-32 in real form, hi and lo BF16 in the K-major
// layout above, 16 KB as 8192 uint16) and the twiddles W1024^(n2 k1) as
// [k1][n2] float2.
void build_tables(uint16_t* b, float2* tw);

}  // namespace tc
}  // namespace psdns
