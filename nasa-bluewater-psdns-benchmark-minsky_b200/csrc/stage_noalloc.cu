// stage_noalloc.cu -- one RK stage without any device allocation.
//
// Some callers cannot call cudaMalloc: a Fortran or OpenACC driver whose
// device arrays are owned by another runtime and that hands us only their
// addresses, or a process started with a fixed device-memory budget handed
// out once at start-up.  psdns_gpu_rk_stage_noalloc serves them: the caller
// passes its own device arrays u and un, and every other piece of device
// memory the stage needs (the transposed cylinder and z-pencil work arrays,
// shift and integrating-factor tables, geometry, twiddles, the velmax
// accumulator) lives in one file-scope static device array of
// PSDNS_NOALLOC_BYTES bytes.  Every GPU that loads the library keeps that
// array until the process exits.
//
// The array's name is only a host-side stand-in for the device address, so
// every call looks the address up with cudaGetSymbolAddress on the current
// device (cheap, and never stale, e.g. after a cudaDeviceReset reloads the
// module).  The call copies its tables from host memory and synchronises the
// caller's stream before it returns, so it refuses a stream that is being
// captured rather than breaking the capture.  All calls share the array and
// it keeps the last call's contents; what must start at zero (the velmax
// accumulator) is cleared by each call.  Calls whose work overlaps on the GPU
// (two streams, or two host threads) race on the array and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "psdns_gpu.h"
#include "psdns_host.h"
#include "stage_kernels.cuh"

namespace psdns {
namespace noalloc {

// largest box the static scratch holds: 64^3 in FP64 (about 16.2 MB of scratch)
constexpr int kMaxN = 64;
constexpr size_t kBytes = PSDNS_NOALLOC_BYTES;

static __device__ __align__(256) unsigned char g_scratch[kBytes];

static size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

// device address of g_scratch on the current device
static int scratch_base(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess) return set_error("cudaGetSymbolAddress(g_scratch) failed: %s", cudaGetErrorString(e));
  *out = (unsigned char*)p;
  return 0;
}

// u and un must be device (or managed) memory of the current device: a host
// pointer or another GPU's memory would reach the kernels otherwise
static int check_device_array(const void* ptr, const char* name) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error("noalloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
  cudaPointerAttributes at;
  e = cudaPointerGetAttributes(&at, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error("noalloc: %s is not a device pointer (%s)", name, cudaGetErrorString(e));
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
    return set_error("noalloc: %s must point to device or managed memory", name);
  if (at.type == cudaMemoryTypeDevice && at.device != dev)
    return set_error("noalloc: %s lives on device %d, the current device is %d", name, at.device, dev);
  return 0;
}

// carve-up of the scratch array for one (n, precision)
struct Plan {
  size_t ub, uz, tabs, colstart, ax, az, kymax, tw, velmax, total;
};

template <typename T, int N>
static Plan plan_for(const Geometry& g) {
  using TL = Tiles<T>;
  const size_t cs = sizeof(C2<T>);
  const size_t nab_i = (g.xz_tot + TL::TB_I - 1) / TL::TB_I, nab_f = (g.xz_tot + TL::TB_F - 1) / TL::TB_F;
  const size_t ub_el = std::max(3 * ubi_var_elems<T>((int)nab_i, N), 4 * ubf_var_elems<T>((int)nab_f, N));
  const size_t uz_el = (size_t)5 * N * N * g.kxn;
  const size_t tab = 2 * (N / 2 + 1 + 2 * N) * cs + (N / 2 + 1 + 2 * N) * sizeof(T);
  Plan p;
  size_t o = 0;
  p.ub = o; o += up256(ub_el * cs);
  p.uz = o; o += up256(uz_el * cs);
  p.tabs = o; o += up256(tab);
  p.colstart = o; o += up256(sizeof(int) * (g.kxn + 1));
  p.ax = o; o += up256(sizeof(int) * g.xz_tot);
  p.az = o; o += up256(sizeof(int) * g.xz_tot);
  p.kymax = o; o += up256(sizeof(int) * g.xz_tot);
  p.tw = o; o += up256(cs * FFTPlan<T, N>::TWSIZE);
  p.velmax = o; o += 256;
  p.total = o;
  return p;
}

template <int N> struct Ls { static constexpr int value = N + N / 32 + 4; };

template <typename T, int N>
static int run(const psdns_params* prm, int kstep, const double* gsh, double dt, C2<T>* u, C2<T>* un,
               double* velmax_out, cudaStream_t st) {
  using C = C2<T>;
  using TL = Tiles<T>;
  Geometry g;
  build_geometry(N, g);
  const Plan pl = plan_for<T, N>(g);
  if (pl.total > kBytes)
    return set_error("noalloc: a %d^3 box needs %zu bytes of scratch, the static array holds %zu", N, pl.total,
                     kBytes);
  unsigned char* base = nullptr;
  if (scratch_base(&base)) return 1;

  // host-side tables: shifts of this stage (shifts.f:146-178), integrating
  // factors (step.f:366-385), twiddles; copied into the scratch array
  const int ks = kstep - 1;
  const double pi = 4. * std::atan(1.);
  const double ph = 2. * pi / N;
  const size_t cs = sizeof(C);
  std::vector<unsigned char> tab(pl.colstart - pl.tabs, 0);
  C* sx = (C*)tab.data();
  C* sy = sx + (N / 2 + 1);
  C* sz = sy + N;
  T* xf = (T*)(tab.data() + 2 * (N / 2 + 1 + 2 * N) * cs);
  T* yf = xf + (N / 2 + 1);
  T* zf = yf + N;
  for (int x = 0; x <= N / 2; x++) {
    const double th = (ph * g.kx[x]) * gsh[0 + 3 * ks];
    sx[x] = cmk<C>((T)std::cos(th), (T)std::sin(th));
  }
  for (int y = 0; y < N; y++) {
    const double th = (ph * g.ky[y]) * gsh[1 + 3 * ks];
    sy[y] = cmk<C>((T)std::cos(th), (T)std::sin(th));
  }
  for (int z = 0; z < N; z++) {
    const double th = (ph * g.kz[z]) * gsh[2 + 3 * ks];
    sz[z] = cmk<C>((T)std::cos(th), (T)std::sin(th));
  }
  const double b11 = prm->beta1 * prm->beta1, b22 = prm->beta2 * prm->beta2, b33 = prm->beta3 * prm->beta3;
  const double nu = prm->viscos;
  double term = b11 * dt;
  for (int x = 0; x <= N / 2; x++) xf[x] = (T)std::exp(-(nu * (g.kx[x] * g.kx[x]) * term));
  term = b22 * dt;
  for (int y = 0; y < N; y++) yf[y] = (T)std::exp(-(nu * (g.ky[y] * g.ky[y]) * term));
  term = b33 * dt;
  for (int z = 0; z < N; z++) zf[z] = (T)std::exp(-(nu * (g.kz[z] * g.kz[z]) * term));
  std::vector<C> tw(FFTPlan<T, N>::TWSIZE);
  build_twiddles<T, N>(tw.data());

#define NA_CK(call)                                                                                   \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return set_error("noalloc: %s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)
  NA_CK(cudaMemcpyAsync(base + pl.tabs, tab.data(), tab.size(), cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(base + pl.colstart, g.colstart.data(), sizeof(int) * (g.kxn + 1), cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(base + pl.ax, g.ax.data(), sizeof(int) * g.xz_tot, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(base + pl.az, g.az.data(), sizeof(int) * g.xz_tot, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(base + pl.kymax, g.kymax.data(), sizeof(int) * g.xz_tot, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(base + pl.tw, tw.data(), cs * tw.size(), cudaMemcpyHostToDevice, st));
  if (kstep == 1) NA_CK(cudaMemsetAsync(base + pl.velmax, 0, sizeof(unsigned long long), st));

  Geo geo;
  geo.n = N; geo.kxn = g.kxn; geo.xz_tot = g.xz_tot; geo.nzt = N / TL::TZ;
  geo.nab_i = (g.xz_tot + TL::TB_I - 1) / TL::TB_I;
  geo.nab_f = (g.xz_tot + TL::TB_F - 1) / TL::TB_F;
  geo.colstart = (const int*)(base + pl.colstart);
  geo.ax = (const int*)(base + pl.ax);
  geo.az = (const int*)(base + pl.az);
  geo.kymax = (const int*)(base + pl.kymax);
  StageTables<T> stb;
  stb.sx = (const C*)(base + pl.tabs);
  stb.sy = stb.sx + (N / 2 + 1);
  stb.sz = stb.sy + N;
  stb.xfac = (const T*)(base + pl.tabs + 2 * (N / 2 + 1 + 2 * N) * cs);
  stb.yfac = stb.xfac + (N / 2 + 1);
  stb.zfac = stb.yfac + N;
  stb.xdif = stb.ydif = stb.zdif = nullptr;   // no scalar on this path
  stb.forc = nullptr;
  stb.kfor = 0; stb.k2fo = 0; stb.kforce2 = 0;
  stb.b11 = (T)b11; stb.b22 = (T)b22; stb.b33 = (T)b33;
  stb.norm = (T)((dt / 2.) / N / N);
  C* ub = (C*)(base + pl.ub);
  C* uz = (C*)(base + pl.uz);
  const C* twd = (const C*)(base + pl.tw);
  unsigned long long* vmx = (unsigned long long*)(base + pl.velmax);
  constexpr int L = Ls<N>::value;
  constexpr size_t TWB = sizeof(C) * FFTPlan<T, N>::TWSIZE;
  const int kxn = g.kxn;
  {
    constexpr int TH = K1Launch<T, N>::THREADS;
    k_yinv<T, N><<<dim3(k1_blocks<T>(geo.nab_i), 3), TH, TWB + sizeof(C) * TL::TB_I * L, st>>>(geo, stb, u, ub, twd);
  }
  {
    constexpr int TH = Launch<T, N, TL::XT2>::THREADS;
    k_zinv<T, N><<<dim3(N, (kxn + TL::XT2 - 1) / TL::XT2, 3), TH, TWB + sizeof(C) * TL::XT2 * L, st>>>(geo, ub, uz,
                                                                                                       twd);
  }
  {
    constexpr int TH = K3Launch<T, N, 0>::THREADS;
    k_xchain<T, N><<<dim3(geo.nzt, N), TH, K3Launch<T, N, 0>::SMEM, st>>>(
        geo, uz, twd, stb.b11, stb.b22, stb.b33, vmx, kstep == 1 ? 1 : 0);
  }
  {
    constexpr int TH = K4Launch<T, N>::THREADS;
    constexpr int XT4 = k4_xt(sizeof(T) == 8, N);
    k_zfwd<T, N><<<dim3(N / TL::YT4, (kxn + XT4 - 1) / XT4), TH, K4Launch<T, N>::SMEM, st>>>(
        geo, uz, ub, twd, stb.b11, stb.b33);
  }
  {
    constexpr int TH = K5Launch<T, N, 0>::THREADS;
    if (kstep == 1)
      k_yfwd<T, N, 1><<<geo.nab_f, TH, TWB + sizeof(C) * 4 * TL::TB_F * L, st>>>(geo, stb, ub, u, un, twd, nullptr);
    else
      k_yfwd<T, N, 2><<<geo.nab_f, TH, TWB + sizeof(C) * 4 * TL::TB_F * L, st>>>(geo, stb, ub, u, un, twd, nullptr);
  }
  NA_CK(cudaGetLastError());
  unsigned long long vm_bits = 0;
  if (kstep == 1) NA_CK(cudaMemcpyAsync(&vm_bits, vmx, sizeof vm_bits, cudaMemcpyDeviceToHost, st));
  // the host tables above must outlive their copies, and velmax must land
  NA_CK(cudaStreamSynchronize(st));
#undef NA_CK
  if (kstep == 1 && velmax_out) std::memcpy(velmax_out, &vm_bits, sizeof(double));
  return 0;
}

}  // namespace noalloc
}  // namespace psdns

using namespace psdns;

extern "C" int psdns_gpu_rk_stage_noalloc(const psdns_params* p, int32_t kstep, const double* gsh, const double* dt,
                                          void* u_dev, void* un_dev, double* velmax_out, void* stream) {
  if (!p || !gsh || !dt || !u_dev || !un_dev) return set_error("noalloc: null argument");
  if (kstep != 1 && kstep != 2) return set_error("noalloc: kstep must be 1 or 2");
  if (!(*dt > 0)) return set_error("noalloc: dt must be positive (pass it at both stages)");
  if (p->nx != p->ny || p->nx != p->nz) return set_error("noalloc: only cubic boxes are supported");
  if (p->nc != 0) return set_error("noalloc: passive scalars are not supported");
  if (p->kforce > 0) return set_error("noalloc: forcing is not supported by this entry point");
  if (p->rkmethod == 4) return set_error("noalloc: this entry point runs the RK2 stages");
  const int n = p->nx;
  if (n > noalloc::kMaxN)
    return set_error("noalloc: grid %d^3 exceeds the largest box the static scratch holds (%d^3)", n,
                     noalloc::kMaxN);
  cudaStream_t st = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    return set_error("noalloc: the stream is not valid on the current device");
  }
  if (cap != cudaStreamCaptureStatusNone)
    return set_error("noalloc: the stream is being captured; this call copies host tables and synchronises the "
                     "stream, so it cannot be captured");
  if (noalloc::check_device_array(u_dev, "u") || noalloc::check_device_array(un_dev, "un")) return 1;
  const bool dbl = p->precision == PSDNS_PREC_FP64;
  if (!dbl && p->precision != PSDNS_PREC_FP32) return set_error("noalloc: bad precision");
#define NA_CASE(NN)                                                                                             \
  case NN:                                                                                                      \
    return dbl ? noalloc::run<double, NN>(p, kstep, gsh, *dt, (double2*)u_dev, (double2*)un_dev, velmax_out, st) \
               : noalloc::run<float, NN>(p, kstep, gsh, *dt, (float2*)u_dev, (float2*)un_dev, velmax_out, st);
  switch (n) {
    NA_CASE(16)
    NA_CASE(32)
    NA_CASE(64)
    default:
      return set_error("noalloc: grid size %d not supported (16, 32 or 64)", n);
  }
#undef NA_CASE
}
