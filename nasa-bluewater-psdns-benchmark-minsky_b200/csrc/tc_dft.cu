// tc_dft.cu -- host tables of the tensor-core DFT, and two C-ABI entry points
// that exercise it on their own: a batched 1-D DFT of lines (FP32 Stockham
// or split-BF16 tensor cores) and a diagnostic of the operand layouts (one
// tcgen05.mma tile).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "psdns_gpu.h"
#include "psdns_host.h"
#include "stage_kernels.cuh"
#include "tc_dft.cuh"

namespace psdns {
namespace tc {

// round to nearest even BF16 (finite values)
static uint16_t f2bf(double v) {
  const float f = (float)v;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
static double bf2d(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

void build_tables(uint16_t* b, float2* tw) {
  const long double pi = 3.14159265358979323846264338327950288L;
  // B[n][k]: n < 32 -> re of output k1 = n, n >= 32 -> im of k1 = n - 32;
  // k < 32 -> re of input n1 = k, k >= 32 -> im of n1 = k - 32.
  // x W32^(n1 k1) = (xr c + xi s) + i (xi c - xr s), c, s of 2 pi n1 k1 / 32
  for (int n = 0; n < 64; n++)
    for (int k = 0; k < 64; k++) {
      const int k1 = n & 31, n1 = k & 31;
      const long double th = 2.0L * pi * (long double)((n1 * k1) % 32) / 32.0L;
      const double c = (double)cosl(th), s = (double)sinl(th);
      const double v = n < 32 ? (k < 32 ? c : s) : (k < 32 ? -s : c);
      const uint16_t hi = f2bf(v), lo = f2bf(v - bf2d(hi));
      b[b_off(n, k) / 2] = hi;
      b[(kBLoOff + b_off(n, k)) / 2] = lo;
    }
  for (int k1 = 0; k1 < 32; k1++)
    for (int n2 = 0; n2 < 32; n2++) {
      const long double th = -2.0L * pi * (long double)(n2 * k1) / 1024.0L;
      tw[k1 * 32 + n2] = make_float2((float)cosl(th), (float)sinl(th));
    }
}

// K-major A layout of the diagnostic (same core-matrix order as B)
__host__ __device__ __forceinline__ constexpr int ak_off(int m, int k) {
  return (m >> 3) * 1024 + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint16_t bf_bits(float v) {
  const __nv_bfloat16_raw h = __nv_bfloat16_raw(__float2bfloat16_rn(v));
  return h.x;
}

// one tile: D (128 x 64) = A (128 x 64) B^T (B given as 64 rows n of 64 k)
__global__ void __launch_bounds__(128) k_tc_gemm_check(const float* __restrict__ a, const float* __restrict__ b,
                                                       float* __restrict__ d, int a_mn, unsigned* err) {
  // A (16 KB) and B (8 KB) at the start of 64 KB and 32 KB regions: the
  // block owns shared memory well past what any reading of the descriptors
  // could reach
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* sa = smem_raw;
  unsigned char* sb = smem_raw + 65536;
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t slot;
  for (int i = threadIdx.x; i < 128 * 64; i += 128) {
    const int m = i >> 6, k = i & 63;
    *reinterpret_cast<uint16_t*>(sa + (a_mn ? a_off(m, k) : ak_off(m, k))) = bf_bits(a[i]);
  }
  for (int i = threadIdx.x; i < 64 * 64; i += 128) {
    const int n = i >> 6, k = i & 63;
    *reinterpret_cast<uint16_t*>(sb + b_off(n, k)) = bf_bits(b[i]);
  }
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  if (threadIdx.x < 32) tmem_alloc<64>(&slot);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = slot;
  if (threadIdx.x == 0) {
    const uint32_t A = smem_u32(sa), B = smem_u32(sb);
    const uint32_t idesc = idesc_bf16(128, 64, a_mn != 0);
    for (int s = 0; s < 4; s++) {
      const uint64_t ad = a_mn ? sdesc(A + s * 4096, 2048, 128) : sdesc(A + s * 256, 128, 1024);
      mma_bf16(tmem, ad, sdesc(B + s * 256, 128, 1024), idesc, s > 0 ? 1u : 0u);
    }
    mma_commit(&bar);
  }
  const bool ok = mbar_wait(&bar, 0);
  if (!ok && (threadIdx.x & 31) == 0) atomicOr(err, 1u);
  fence_after();
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float v[32];
  for (int h = 0; h < 2; h++) {
    tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 32 * h, v);
    for (int c = 0; c < 32; c++) d[(32 * q + lane) * 64 + 32 * h + c] = v[c];
  }
  fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after();
    tmem_free<64>(tmem);
  }
}

// batched forward DFT of 1024-point lines, 8 lines per block (one warp each)
template <int MODE>
__global__ void __launch_bounds__(256) k_dft_lines(const float2* __restrict__ in, float2* __restrict__ out,
                                                   long long nlines, const float2* __restrict__ tw_g,
                                                   const uint4* __restrict__ btab, const float2* __restrict__ tw2,
                                                   unsigned* err) {
  constexpr int N = 1024, NL = 8, THREADS = 256, L = LS<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tws = reinterpret_cast<float2*>(smem_raw);
  float2* buf = tws + FFTPlan<float, N>::TWSIZE;
  unsigned char* bsm = reinterpret_cast<unsigned char*>(buf + NL * L);
  uint64_t* bar = reinterpret_cast<uint64_t*>(bsm + kBBytes);
  uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
  const long long l0 = (long long)blockIdx.x * NL;
  const int nl = (int)(nlines - l0 < NL ? nlines - l0 : NL);
  for (int e = threadIdx.x; e < nl * N; e += THREADS) {
    const int l = e / N, i = e % N;
    buf[l * L + pad32(i)] = in[(l0 + l) * N + i];
  }
  if constexpr (MODE == 0) {
    load_twiddles<float, N>(tws, tw_g);
    cp_async_wait_all();
    __syncthreads();
    fft_lines<float, N, THREADS>(buf, nl, L, tws);
  } else {
    Work w;
    setup<128>(w, bsm, bar, slot, btab, tw2, err);
    fft1024_lines<THREADS>(buf, nl, L, w);
    teardown<128>(w);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nl * N; e += THREADS) {
    const int l = e / N, i = e % N;
    out[(l0 + l) * N + i] = buf[l * L + pad32(i)];
  }
}

constexpr size_t dft_smem() {
  return sizeof(float2) * (FFTPlan<float, 1024>::TWSIZE + 8 * LS<1024>::value) + kBBytes + 16;
}

}  // namespace tc
}  // namespace psdns

using namespace psdns;

#define TC_CK(call)                                                                                          \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess) { rc = set_error("%s failed: %s", #call, cudaGetErrorString(e_)); goto done; }   \
  } while (0)

extern "C" int psdns_gpu_tc_gemm_check(int32_t a_mn_major, const float* a, const float* b, float* d) {
  if (!a || !b || !d) return set_error("tc_gemm_check: null argument");
  int rc = 0;
  float *da = nullptr, *db = nullptr, *dd = nullptr;
  unsigned* derr = nullptr;
  unsigned herr = 0;
  TC_CK(cudaMalloc(&da, sizeof(float) * 128 * 64));
  TC_CK(cudaMalloc(&db, sizeof(float) * 64 * 64));
  TC_CK(cudaMalloc(&dd, sizeof(float) * 128 * 64));
  TC_CK(cudaMalloc(&derr, sizeof(unsigned)));
  TC_CK(cudaMemset(derr, 0, sizeof(unsigned)));
  TC_CK(cudaMemcpy(da, a, sizeof(float) * 128 * 64, cudaMemcpyHostToDevice));
  TC_CK(cudaMemcpy(db, b, sizeof(float) * 64 * 64, cudaMemcpyHostToDevice));
  TC_CK(cudaFuncSetAttribute(tc::k_tc_gemm_check, cudaFuncAttributeMaxDynamicSharedMemorySize, 98304));
  tc::k_tc_gemm_check<<<1, 128, 98304>>>(da, db, dd, a_mn_major ? 1 : 0, derr);
  TC_CK(cudaGetLastError());
  TC_CK(cudaMemcpy(d, dd, sizeof(float) * 128 * 64, cudaMemcpyDeviceToHost));
  TC_CK(cudaMemcpy(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (herr) rc = set_error("tc_gemm_check: the MMA completion wait ran out (error word %u)", herr);
done:
  cudaFree(da); cudaFree(db); cudaFree(dd); cudaFree(derr);
  return rc;
}

extern "C" int psdns_gpu_dft_lines(int32_t n, int64_t nlines, int32_t mode, const double* in, double* out) {
  if (!in || !out) return set_error("dft_lines: null argument");
  if (n != 1024) return set_error("dft_lines: n must be 1024");
  if (nlines <= 0 || nlines > (1LL << 22)) return set_error("dft_lines: nlines must be in 1 .. 2^22");
  if (mode != 0 && mode != 1) return set_error("dft_lines: mode must be 0 (FP32) or 1 (tensor cores)");
  int rc = 0;
  const size_t cnt = (size_t)nlines * n;
  std::vector<float2> h(cnt);
  for (size_t i = 0; i < cnt; i++) h[i] = make_float2((float)in[2 * i], (float)in[2 * i + 1]);
  std::vector<float2> tw(FFTPlan<float, 1024>::TWSIZE), tw2(1024);
  std::vector<uint16_t> bt(tc::kBBytes / 2);
  build_twiddles<float, 1024>(tw.data());
  tc::build_tables(bt.data(), tw2.data());
  float2 *din = nullptr, *dout = nullptr, *dtw = nullptr, *dtw2 = nullptr;
  void* dbt = nullptr;
  unsigned* derr = nullptr;
  unsigned herr = 0;
  const size_t smem = tc::dft_smem();
  const int blocks = (int)((nlines + 7) / 8);
  TC_CK(cudaMalloc(&din, sizeof(float2) * cnt));
  TC_CK(cudaMalloc(&dout, sizeof(float2) * cnt));
  TC_CK(cudaMalloc(&dtw, sizeof(float2) * tw.size()));
  TC_CK(cudaMalloc(&dtw2, sizeof(float2) * tw2.size()));
  TC_CK(cudaMalloc(&dbt, tc::kBBytes));
  TC_CK(cudaMalloc(&derr, sizeof(unsigned)));
  TC_CK(cudaMemset(derr, 0, sizeof(unsigned)));
  TC_CK(cudaMemcpy(din, h.data(), sizeof(float2) * cnt, cudaMemcpyHostToDevice));
  TC_CK(cudaMemcpy(dtw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice));
  TC_CK(cudaMemcpy(dtw2, tw2.data(), sizeof(float2) * tw2.size(), cudaMemcpyHostToDevice));
  TC_CK(cudaMemcpy(dbt, bt.data(), tc::kBBytes, cudaMemcpyHostToDevice));
  if (mode == 0) {
    TC_CK(cudaFuncSetAttribute(tc::k_dft_lines<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    tc::k_dft_lines<0><<<blocks, 256, smem>>>(din, dout, nlines, dtw, (const uint4*)dbt, dtw2, derr);
  } else {
    TC_CK(cudaFuncSetAttribute(tc::k_dft_lines<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    tc::k_dft_lines<1><<<blocks, 256, smem>>>(din, dout, nlines, dtw, (const uint4*)dbt, dtw2, derr);
  }
  TC_CK(cudaGetLastError());
  TC_CK(cudaMemcpy(h.data(), dout, sizeof(float2) * cnt, cudaMemcpyDeviceToHost));
  TC_CK(cudaMemcpy(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (herr) rc = set_error("dft_lines: an MMA completion wait ran out (error word %u)", herr);
  for (size_t i = 0; i < cnt; i++) {
    out[2 * i] = h[i].x;
    out[2 * i + 1] = h[i].y;
  }
done:
  cudaFree(din); cudaFree(dout); cudaFree(dtw); cudaFree(dtw2); cudaFree(dbt); cudaFree(derr);
  return rc;
}
