// learned.cu -- the spectral-correction network of the learned coarse solver:
// a multilayer perceptron with BF16 weights and FP32 accumulation, trained on
// the device by its own forward, backward and Adam kernels.
//
// The network maps per-shell features of a coarse-grid spectrum to an eddy
// viscosity: g = softplus(W3 tanh(W2 tanh(W1 tanh(W0 x + b0) + b1) + b2) + b3)
// (four layers: NF -> H -> H -> H -> 1), nu_t(k) = nu g.  It has no
// counterpart in the reference (which only runs the resolved DNS); the
// quantities it is trained and judged on are the reference's statistics:
// E(k) and epsilon of sptr.f:354-365 and the du/dx moments of vgmomt.f.
//
// Training loss (full batch): L = sum_i w_i (a_i g_i - tau_i)^2 / sum_i w_i,
// with a_i = 2 nu k_i^2 Delta (the log-energy damping that nu_t causes over
// Delta) and tau_i = ln(E_coarse(k_i) / E_filtered(k_i)) the damping that
// would bring the coarse run's shell energy onto the filtered fine run's.
//
// Parameters: FP32 master copy (Adam state beside it) and a BF16 copy that
// every forward pass reads; activations and accumulation are FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "psdns_gpu.h"
#include "psdns_host.h"

namespace psdns {
namespace mlp {

constexpr int NF = PSDNS_CORRECTOR_FEATURES;   // input features
constexpr int H = PSDNS_CORRECTOR_WIDTH;       // hidden width
// flat parameter vector: W0[H][NF] b0[H] W1[H][H] b1[H] W2[H][H] b2[H] W3[H] b3
constexpr int OW0 = 0, OB0 = OW0 + H * NF, OW1 = OB0 + H, OB1 = OW1 + H * H, OW2 = OB1 + H, OB2 = OW2 + H * H,
              OW3 = OB2 + H, OB3 = OW3 + H, NP = OB3 + 1;
constexpr int BLOCK = 128;

__device__ __forceinline__ float softplus(float z) { return z > 20.f ? z : log1pf(__expf(z)); }
__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + __expf(-z)); }

__device__ __forceinline__ float bf16_to_f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// stage the BF16 weights into shared memory as floats
__device__ __forceinline__ void load_weights(float* ws, const uint16_t* __restrict__ wb) {
  for (int i = threadIdx.x; i < NP; i += blockDim.x) ws[i] = bf16_to_f(wb[i]);
  __syncthreads();
}

// forward pass of one sample; keeps the hidden activations
__device__ __forceinline__ float forward(const float* w, const float* x, float* a1, float* a2, float* a3, float& z) {
#pragma unroll 4
  for (int j = 0; j < H; j++) {
    float s = w[OB0 + j];
#pragma unroll
    for (int i = 0; i < NF; i++) s = fmaf(w[OW0 + j * NF + i], x[i], s);
    a1[j] = tanhf(s);
  }
#pragma unroll 4
  for (int j = 0; j < H; j++) {
    float s = w[OB1 + j];
#pragma unroll
    for (int i = 0; i < H; i++) s = fmaf(w[OW1 + j * H + i], a1[i], s);
    a2[j] = tanhf(s);
  }
#pragma unroll 4
  for (int j = 0; j < H; j++) {
    float s = w[OB2 + j];
#pragma unroll
    for (int i = 0; i < H; i++) s = fmaf(w[OW2 + j * H + i], a2[i], s);
    a3[j] = tanhf(s);
  }
  float s = w[OB3];
#pragma unroll
  for (int i = 0; i < H; i++) s = fmaf(w[OW3 + i], a3[i], s);
  z = s;
  return softplus(s);
}

__global__ void __launch_bounds__(BLOCK) k_forward(const uint16_t* __restrict__ wb, const float* __restrict__ x,
                                                   long long nb, float* __restrict__ g) {
  __shared__ float ws[NP];
  load_weights(ws, wb);
  float a1[H], a2[H], a3[H], xi[NF], z;
  for (long long s = blockIdx.x * (long long)BLOCK + threadIdx.x; s < nb; s += (long long)gridDim.x * BLOCK) {
#pragma unroll
    for (int i = 0; i < NF; i++) xi[i] = x[s * NF + i];
    g[s] = forward(ws, xi, a1, a2, a3, z);
  }
}

// loss and its gradient with respect to the parameters (summed into grad,
// which the caller zeroes); loss_sum gets sum_i w_i (a_i g_i - tau_i)^2
__global__ void __launch_bounds__(BLOCK) k_grad(const uint16_t* __restrict__ wb, const float* __restrict__ x,
                                                const float* __restrict__ a, const float* __restrict__ tau,
                                                const float* __restrict__ wt, long long nb, float inv_wsum,
                                                float* __restrict__ grad, double* __restrict__ loss_sum) {
  __shared__ float ws[NP];
  __shared__ float gs[NP];
  for (int i = threadIdx.x; i < NP; i += BLOCK) gs[i] = 0.f;
  load_weights(ws, wb);
  float a1[H], a2[H], a3[H], xi[NF], d[H], e[H], z;
  double lsum = 0.0;
  for (long long s = blockIdx.x * (long long)BLOCK + threadIdx.x; s < nb; s += (long long)gridDim.x * BLOCK) {
#pragma unroll
    for (int i = 0; i < NF; i++) xi[i] = x[s * NF + i];
    const float gv = forward(ws, xi, a1, a2, a3, z);
    const float r = a[s] * gv - tau[s];
    lsum += (double)wt[s] * r * r;
    // dL/dz
    const float dz = 2.f * wt[s] * inv_wsum * a[s] * r * sigmoid(z);
    atomicAdd(&gs[OB3], dz);
#pragma unroll 4
    for (int i = 0; i < H; i++) {
      atomicAdd(&gs[OW3 + i], dz * a3[i]);
      d[i] = dz * ws[OW3 + i] * (1.f - a3[i] * a3[i]);   // dL/d(pre-activation of layer 3)
    }
    // layer 2: W2 [H][H] acts on a2
#pragma unroll 2
    for (int j = 0; j < H; j++) {
      atomicAdd(&gs[OB2 + j], d[j]);
      for (int i = 0; i < H; i++) atomicAdd(&gs[OW2 + j * H + i], d[j] * a2[i]);
    }
#pragma unroll 4
    for (int i = 0; i < H; i++) {
      float t = 0.f;
      for (int j = 0; j < H; j++) t = fmaf(ws[OW2 + j * H + i], d[j], t);
      e[i] = t * (1.f - a2[i] * a2[i]);
    }
#pragma unroll 2
    for (int j = 0; j < H; j++) {
      atomicAdd(&gs[OB1 + j], e[j]);
      for (int i = 0; i < H; i++) atomicAdd(&gs[OW1 + j * H + i], e[j] * a1[i]);
    }
#pragma unroll 4
    for (int i = 0; i < H; i++) {
      float t = 0.f;
      for (int j = 0; j < H; j++) t = fmaf(ws[OW1 + j * H + i], e[j], t);
      d[i] = t * (1.f - a1[i] * a1[i]);
    }
#pragma unroll 2
    for (int j = 0; j < H; j++) {
      atomicAdd(&gs[OB0 + j], d[j]);
#pragma unroll
      for (int i = 0; i < NF; i++) atomicAdd(&gs[OW0 + j * NF + i], d[j] * xi[i]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NP; i += BLOCK)
    if (gs[i] != 0.f) atomicAdd(grad + i, gs[i]);
  // block sum of the loss
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((threadIdx.x & 31) == 0 && lsum != 0.0) atomicAdd(loss_sum, lsum);
}

// one Adam step on the FP32 master weights; refreshes the BF16 copy and
// zeroes the gradient for the next step
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, uint16_t* __restrict__ wb,
                       float* __restrict__ g, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NP) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  const __nv_bfloat16_raw h = __nv_bfloat16_raw(__float2bfloat16_rn(wi));
  wb[i] = h.x;
  g[i] = 0.f;
}

__global__ void k_to_bf16(const float* __restrict__ w, uint16_t* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NP) return;
  const __nv_bfloat16_raw h = __nv_bfloat16_raw(__float2bfloat16_rn(w[i]));
  wb[i] = h.x;
}

struct Corrector {
  float *d_w = nullptr, *d_m = nullptr, *d_v = nullptr, *d_g = nullptr;
  uint16_t* d_wb = nullptr;
  double* d_loss = nullptr;
  float *d_x = nullptr, *d_a = nullptr, *d_tau = nullptr, *d_wt = nullptr, *d_out = nullptr;
  long long cap = 0;
  long long adam_t = 0;
  cudaStream_t stream = nullptr;
};

#define ML_CK(call)                                                                         \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return set_error("corrector: %s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

static int ensure_batch(Corrector& c, long long nb) {
  if (nb <= c.cap) return 0;
  cudaFree(c.d_x); cudaFree(c.d_a); cudaFree(c.d_tau); cudaFree(c.d_wt); cudaFree(c.d_out);
  c.d_x = c.d_a = c.d_tau = c.d_wt = c.d_out = nullptr;
  c.cap = 0;
  ML_CK(cudaMalloc(&c.d_x, sizeof(float) * NF * nb));
  ML_CK(cudaMalloc(&c.d_a, sizeof(float) * nb));
  ML_CK(cudaMalloc(&c.d_tau, sizeof(float) * nb));
  ML_CK(cudaMalloc(&c.d_wt, sizeof(float) * nb));
  ML_CK(cudaMalloc(&c.d_out, sizeof(float) * nb));
  c.cap = nb;
  return 0;
}

static int grid_for(long long nb) { return (int)std::min<long long>((nb + BLOCK - 1) / BLOCK, 148 * 4); }

// splitmix64, for reproducible initial weights
static uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int forward_host(void* corr, long long nb, const float* x, float* g) {
  Corrector& c = *(Corrector*)corr;
  if (ensure_batch(c, nb)) return 1;
  ML_CK(cudaMemcpyAsync(c.d_x, x, sizeof(float) * NF * nb, cudaMemcpyHostToDevice, c.stream));
  k_forward<<<grid_for(nb), BLOCK, 0, c.stream>>>(c.d_wb, c.d_x, nb, c.d_out);
  ML_CK(cudaGetLastError());
  ML_CK(cudaMemcpyAsync(g, c.d_out, sizeof(float) * nb, cudaMemcpyDeviceToHost, c.stream));
  ML_CK(cudaStreamSynchronize(c.stream));
  return 0;
}

static int upload_batch(Corrector& c, long long nb, const float* x, const float* a, const float* tau,
                        const float* wt, float& inv_wsum) {
  if (ensure_batch(c, nb)) return 1;
  double ws = 0;
  for (long long i = 0; i < nb; i++) ws += wt[i];
  if (!(ws > 0)) return set_error("corrector: the sample weights sum to zero");
  inv_wsum = (float)(1.0 / ws);
  ML_CK(cudaMemcpyAsync(c.d_x, x, sizeof(float) * NF * nb, cudaMemcpyHostToDevice, c.stream));
  ML_CK(cudaMemcpyAsync(c.d_a, a, sizeof(float) * nb, cudaMemcpyHostToDevice, c.stream));
  ML_CK(cudaMemcpyAsync(c.d_tau, tau, sizeof(float) * nb, cudaMemcpyHostToDevice, c.stream));
  ML_CK(cudaMemcpyAsync(c.d_wt, wt, sizeof(float) * nb, cudaMemcpyHostToDevice, c.stream));
  return 0;
}

}  // namespace mlp
}  // namespace psdns

using namespace psdns;
using namespace psdns::mlp;

extern "C" {

int psdns_gpu_corrector_create(int32_t seed, void** out) {
  if (!out) return set_error("corrector: null argument");
  *out = nullptr;
  Corrector* c = new Corrector();
  auto fail = [&](int rc) { psdns_gpu_corrector_destroy(c); return rc; };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error("corrector: stream creation failed"));
  if (cudaMalloc(&c->d_w, sizeof(float) * NP) != cudaSuccess || cudaMalloc(&c->d_m, sizeof(float) * NP) != cudaSuccess ||
      cudaMalloc(&c->d_v, sizeof(float) * NP) != cudaSuccess || cudaMalloc(&c->d_g, sizeof(float) * NP) != cudaSuccess ||
      cudaMalloc(&c->d_wb, sizeof(uint16_t) * NP) != cudaSuccess || cudaMalloc(&c->d_loss, sizeof(double)) != cudaSuccess)
    return fail(set_error("corrector: cudaMalloc failed"));
  // Glorot-uniform weights, zero biases
  std::vector<float> w(NP, 0.f);
  uint64_t s = (uint64_t)(uint32_t)seed * 0x2545F4914F6CDD1Dull + 1;
  auto fill = [&](int off, int fan_out, int fan_in) {
    const double r = std::sqrt(6.0 / (fan_in + fan_out));
    for (int i = 0; i < fan_out * fan_in; i++)
      w[off + i] = (float)((2.0 * ((splitmix(s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0) * r);
  };
  fill(OW0, H, NF);
  fill(OW1, H, H);
  fill(OW2, H, H);
  fill(OW3, 1, H);
  if (psdns_gpu_corrector_params(c, 0, w.data())) return fail(1);
  *out = c;
  return 0;
}

int psdns_gpu_corrector_destroy(void* corr) {
  Corrector* c = (Corrector*)corr;
  if (!c) return 0;
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* p[] = {c->d_w, c->d_m, c->d_v, c->d_g, c->d_wb, c->d_loss, c->d_x, c->d_a, c->d_tau, c->d_wt, c->d_out};
  for (void* q : p)
    if (q) cudaFree(q);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int psdns_gpu_corrector_params(void* corr, int32_t get, float* w) {
  Corrector* c = (Corrector*)corr;
  if (!c || !w) return set_error("corrector: null argument");
  if (get) {
    ML_CK(cudaMemcpyAsync(w, c->d_w, sizeof(float) * NP, cudaMemcpyDeviceToHost, c->stream));
  } else {
    ML_CK(cudaMemcpyAsync(c->d_w, w, sizeof(float) * NP, cudaMemcpyHostToDevice, c->stream));
    ML_CK(cudaMemsetAsync(c->d_m, 0, sizeof(float) * NP, c->stream));
    ML_CK(cudaMemsetAsync(c->d_v, 0, sizeof(float) * NP, c->stream));
    ML_CK(cudaMemsetAsync(c->d_g, 0, sizeof(float) * NP, c->stream));
    k_to_bf16<<<(NP + 255) / 256, 256, 0, c->stream>>>(c->d_w, c->d_wb);
    ML_CK(cudaGetLastError());
    c->adam_t = 0;
  }
  ML_CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int psdns_gpu_corrector_forward(void* corr, int64_t nb, const float* x, float* g) {
  if (!corr || !x || !g || nb <= 0) return set_error("corrector: bad argument");
  return forward_host(corr, nb, x, g);
}

int psdns_gpu_corrector_grad(void* corr, int64_t nb, const float* x, const float* a, const float* tau,
                             const float* wt, float* grad, double* loss) {
  Corrector* c = (Corrector*)corr;
  if (!c || !x || !a || !tau || !wt || !grad || !loss || nb <= 0) return set_error("corrector: bad argument");
  float inv = 0.f;
  if (upload_batch(*c, nb, x, a, tau, wt, inv)) return 1;
  ML_CK(cudaMemsetAsync(c->d_g, 0, sizeof(float) * NP, c->stream));
  ML_CK(cudaMemsetAsync(c->d_loss, 0, sizeof(double), c->stream));
  k_grad<<<grid_for(nb), BLOCK, 0, c->stream>>>(c->d_wb, c->d_x, c->d_a, c->d_tau, c->d_wt, nb, inv, c->d_g,
                                                c->d_loss);
  ML_CK(cudaGetLastError());
  ML_CK(cudaMemcpyAsync(grad, c->d_g, sizeof(float) * NP, cudaMemcpyDeviceToHost, c->stream));
  ML_CK(cudaMemcpyAsync(loss, c->d_loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ML_CK(cudaMemsetAsync(c->d_g, 0, sizeof(float) * NP, c->stream));
  ML_CK(cudaStreamSynchronize(c->stream));
  *loss *= (double)inv;
  return 0;
}

int psdns_gpu_corrector_train(void* corr, int64_t nb, const float* x, const float* a, const float* tau,
                              const float* wt, int32_t iters, double lr, double* loss_hist) {
  Corrector* c = (Corrector*)corr;
  if (!c || !x || !a || !tau || !wt || nb <= 0 || iters <= 0 || !(lr > 0)) return set_error("corrector: bad argument");
  float inv = 0.f;
  if (upload_batch(*c, nb, x, a, tau, wt, inv)) return 1;
  std::vector<double> hist(iters, 0.0);
  double* d_hist = nullptr;
  ML_CK(cudaMalloc(&d_hist, sizeof(double) * iters));
  int rc = 0;
  if (cudaMemsetAsync(d_hist, 0, sizeof(double) * iters, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_g, 0, sizeof(float) * NP, c->stream) != cudaSuccess)
    rc = set_error("corrector: memset failed");
  const float b1 = 0.9f, b2 = 0.999f;
  for (int it = 0; it < iters && !rc; it++) {
    k_grad<<<grid_for(nb), BLOCK, 0, c->stream>>>(c->d_wb, c->d_x, c->d_a, c->d_tau, c->d_wt, nb, inv, c->d_g,
                                                  d_hist + it);
    c->adam_t++;
    const float c1 = 1.f - std::pow(b1, (float)c->adam_t), c2 = 1.f - std::pow(b2, (float)c->adam_t);
    k_adam<<<(NP + 255) / 256, 256, 0, c->stream>>>(c->d_w, c->d_m, c->d_v, c->d_wb, c->d_g, (float)lr, b1, b2,
                                                    1e-8f, c1, c2);
    if (cudaGetLastError() != cudaSuccess) rc = set_error("corrector: training launch failed");
  }
  if (!rc && (cudaMemcpyAsync(hist.data(), d_hist, sizeof(double) * iters, cudaMemcpyDeviceToHost, c->stream) !=
                  cudaSuccess ||
              cudaStreamSynchronize(c->stream) != cudaSuccess))
    rc = set_error("corrector: reading the loss history failed");
  cudaFree(d_hist);
  if (!rc && loss_hist)
    for (int i = 0; i < iters; i++) loss_hist[i] = hist[i] * inv;
  return rc;
}

}  // extern "C"
