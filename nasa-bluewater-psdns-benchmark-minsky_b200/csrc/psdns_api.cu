// psdns_api.cu -- host side of libpsdns_gpu: the C-ABI of include/psdns_gpu.h.
//
// Host responsibilities mirror the parts of the reference driver that stay on
// the CPU: the cylinder geometry and mask (PSDNS/mpisetup.f:307-357,
// PSDNS/masks.f), the grid-shift random numbers (PSDNS/shifts.f with
// PSDNS/ranu.f, PSDNS/ranseq.f), the time-step control and integrating
// factors (PSDNS/step.f) and the forcing table (PSDNS/force.f).  Everything
// proportional to the grid runs in the kernels of stage_kernels.cuh.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "psdns_gpu.h"
#include "psdns_host.h"
#include "stage_kernels.cuh"
#include "field_init.cuh"
#include "spectra.cuh"
#include "learned.cuh"

namespace psdns {

#ifndef PSDNS_INST_N
static thread_local std::string g_last_error;

int set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return 1;
}

#endif

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#ifndef PSDNS_INST_N

// ---------------------------------------------------------------------------
// geometry (PSDNS/mpisetup.f:307-357, next_xz :710-732, masks.f:46-83)
// ---------------------------------------------------------------------------
void build_geometry(int n, Geometry& g) {
  g.n = n;
  g.kx.resize(n / 2 + 1);
  g.ky.resize(n);
  g.kz.resize(n);
  for (int x = 0; x <= n / 2; x++) g.kx[x] = x;
  for (int y = 0; y < n; y++) g.ky[y] = (y > n / 2) ? y - n : y;
  for (int z = 0; z < n; z++) g.kz[z] = (z > n / 2) ? z - n : z;
  // kxn = min(n/2, (int)(n sqrt(2)/3) + 1) (init.f:29), in integer
  // arithmetic so that the kernels can use it as a compile-time constant
  const int kxn = kxn_of(n);
  g.kxn = kxn;
  g.cut.assign(kxn, 0);
  g.colstart.assign(kxn + 1, 0);
  const double rnxi = 1.0 / n;
  int tot = 0;
  for (int x = 0; x < kxn; x++) {
    const double t = g.kx[x] * rnxi;
    const double rc = n * (1.0 - 2.0 * std::sqrt(2.0 / 9.0 - t * t));
    const int c = (int)(rc / 2);
    g.cut[x] = c;
    g.colstart[x] = tot;
    tot += n - 1 - c * 2;
  }
  g.colstart[kxn] = tot;
  g.xz_tot = tot;
  g.ax.resize(tot);
  g.az.resize(tot);
  g.kymax.resize(tot);
  const double two9 = 2. / 9., rnyi = 1. / n, rnzi = 1. / n;
  for (int x = 0; x < kxn; x++) {
    const int kcx = n / 2 - 1 - g.cut[x];
    for (int i = 0; i < 2 * kcx + 1; i++) {
      const int a = g.colstart[x] + i;
      const int kz = (i <= kcx) ? i : i - (2 * kcx + 1);
      const int z = kz < 0 ? kz + n : kz;
      g.ax[a] = x;
      g.az[a] = z;
      // volatile keeps each product rounded on its own (no contraction)
      volatile double tx = g.kx[x] * rnxi;
      volatile double sqkx = tx * tx;
      volatile double tz = g.kz[z] * rnzi;
      volatile double tz2 = tz * tz;
      volatile double sqkz = tz2 + sqkx;
      int km = -1;
      for (int m = 0; m <= n / 2; m++) {
        volatile double ty = m * rnyi;
        volatile double ty2 = ty * ty;
        volatile double sqk = ty2 + sqkz;
        if (sqk > two9) break;
        km = m;
      }
      g.kymax[a] = km;
    }
  }
}

// ---------------------------------------------------------------------------
// random numbers (PSDNS/ranu.f:27-29, PSDNS/ranseq.f:62-141)
// ---------------------------------------------------------------------------
void Rng::init(int32_t seed) {
  for (int i = 0; i < 20; i++) iseq[i] = 0;
  klast = 1;
  iseed = 0;
  ifst = 0;
  seed_input = seed;
}
void Rng::ranseq(int k) {
  if (ifst == 0) {
    ifst = 1;
    for (int i = 0; i < 20; i++) iseq[i] = seed_input;
    klast = 1;
    iseed = iseq[0];
  }
  iseq[klast - 1] = iseed;
  klast = k;
  iseed = iseq[k - 1];
}
double Rng::ranu() {
  uint32_t s = (uint32_t)iseed * 65539u;
  int32_t is = (int32_t)s;
  if (is < 0) is = (int32_t)((uint32_t)is + 2147483647u + 1u);
  iseed = is;
  return (double)is * 0.46566127e-9;
}

#endif  // PSDNS_INST_N

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct Ctx {
  psdns_params p;
  Geometry g;
  int n, prec, nzt, nab_i, nab_f;
  int nc = 0, nv = 3;   // passive scalars and stored variables (3 + nc)
  size_t csz;  // sizeof complex element on device
  int *d_colstart = nullptr, *d_ax = nullptr, *d_az = nullptr, *d_kymax = nullptr;
  void *d_tw = nullptr, *d_tabs = nullptr, *d_u = nullptr, *d_un = nullptr, *d_ub = nullptr, *d_uz = nullptr;
  void *d_forc = nullptr;
  double* d_efkz = nullptr;
  // tensor-core transforms (dft = PSDNS_DFT_TC_BF16X3): B operands,
  // twiddles and the error word of the bounded MMA waits
  int dft = PSDNS_DFT_FP32;
  void* d_tcb = nullptr;
  float2* d_tw2 = nullptr;
  unsigned* d_tcerr = nullptr;
  double* d_shf = nullptr;   // per-shell factors of the learned correction
  // RK scheme (timestep_module.f:295-308): 2 (proc4a/proc4b) or 4
  // (advanc_1..4, accumulator u1 of comp_set.f:72 in d_u1)
  int rk = 2;
  void* d_u1 = nullptr;
  unsigned long long* d_velmax = nullptr;
  void* h_tabs = nullptr;          // pinned staging of the stage tables
  unsigned long long* h_velmax = nullptr;
  cudaStream_t stream = nullptr;
  size_t ub_elems = 0, uz_elems = 0, st_elems = 0;
  // stepping state
  Rng rng;
  double gsh[3][2] = {{0, 0}, {0, 0}, {0, 0}}, gsh4[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  int jstep = 0;
  double time = 0, dt = 0, dt0 = 0, dt2 = 0, velmax = 0;
  // > 0 after a restart from chkptin/ranin (store.f icall 3): the first
  // step draws no initial gsh(:,2) (shifts.f:47) and the forcing keeps the
  // restored processes (vfuo.f, vfiuo.f: istart > 0)
  int istart = 0;
  int kfor = 0, k2fo = 0;
  EPForcing forcing;
  // Lagrangian particles (positions/velocities FP64, spline coefficients in
  // the state precision, interleaved as 4-vectors [y][z][x])
  long long np = 0;
  double *d_pos = nullptr, *d_vel = nullptr;
  void *d_bs = nullptr, *d_spf = nullptr;
  bool part_first = true;
  long long pin_nop = 0;           // partin request, made at the first particle phase
  int pin_pstart = 0, pin_kipran = 11;
  void* h_forc = nullptr;          // pinned staging of the forcing table (device precision)
  std::vector<double> efk_host;    // energy input per shell of the last step (forcdt.f)
  double erate = 0, eirate[3] = {0, 0, 0};
  // per-kernel CUDA-event timing: [stage][kernel][begin/end]
  bool prof = false;
  cudaEvent_t ev[4][6][2] = {};   // RK4 has four stages
  // asynchronous state copies: copy streams, complex(8) staging of the whole
  // state in each direction, per-chunk events (allocated on first use)
  static constexpr int kChunks = 12;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  void *d_in_stage = nullptr, *d_out_stage = nullptr;
  cudaEvent_t ev_h2d[kChunks] = {}, ev_conv_in[kChunks] = {}, ev_conv_out[kChunks] = {}, ev_d2h[kChunks] = {};
  const char* pend_out = nullptr;    // host range of the last get_state_async
  size_t pend_out_bytes = 0;
  bool in_pending = false;
  // sphere-only copies (pinned host memory read and written by kernels):
  // the downloads run on s_out after ev_ready; an upload that directly
  // follows a download waits for it chunk by chunk
  cudaEvent_t ev_ready = nullptr;
  long long api_calls = 0, sphere_get_call = -1;
  bool sphere_get_pending = false;
  bool pend_sphere = false;          // the pending download was a sphere copy
  double prof_ms[6] = {0, 0, 0, 0, 0, 0};
  long long prof_n[6] = {0, 0, 0, 0, 0, 0};
  bool prof_pending[4] = {false, false, false, false};
};

static void prof_mark(Ctx& c, int stage, int k, int end) {
  if (c.prof) cudaEventRecord(c.ev[stage][k][end], c.stream);
}

// fold the events of a finished stage into the totals (stream already synced)
static void prof_collect(Ctx& c, int stage, int k0, int k1) {
  if (!c.prof) return;
  for (int k = k0; k < k1; k++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c.ev[stage][k][0], c.ev[stage][k][1]) == cudaSuccess) {
      c.prof_ms[k] += ms;
      c.prof_n[k] += 1;
    }
  }
}

template <typename T> struct TabLayout {
  // offsets in bytes inside the stage-table block
  size_t sx[2], sy[2], sz[2], xf, yf, zf, xd, yd, zd, total;
  explicit TabLayout(int n) {
    const size_t c = sizeof(C2<T>), r = sizeof(T);
    size_t o = 0;
    for (int k = 0; k < 2; k++) { sx[k] = o; o += c * (n / 2 + 1); }
    for (int k = 0; k < 2; k++) { sy[k] = o; o += c * n; }
    for (int k = 0; k < 2; k++) { sz[k] = o; o += c * n; }
    xf = o; o += r * (n / 2 + 1);
    yf = o; o += r * n;
    zf = o; o += r * n;
    xd = o; o += r * (n / 2 + 1);
    yd = o; o += r * n;
    zd = o; o += r * n;
    total = (o + 255) & ~size_t(255);
  }
};

// complex elements of one variable in the full half-complex layout
static size_t full_elems(const Ctx& c) { return (size_t)(c.n / 2 + 1) * c.n * c.n; }

static Geo make_geo(const Ctx& c) {
  Geo g;
  g.n = c.n; g.kxn = c.g.kxn; g.xz_tot = c.g.xz_tot; g.nzt = c.nzt;
  g.nab_i = c.nab_i; g.nab_f = c.nab_f;
  g.colstart = c.d_colstart; g.ax = c.d_ax; g.az = c.d_az; g.kymax = c.d_kymax;
  return g;
}

template <typename T>
static StageTables<T> make_tables(const Ctx& c, int ks) {
  TabLayout<T> L(c.n);
  const char* b = (const char*)c.d_tabs;
  StageTables<T> st;
  st.sx = (const C2<T>*)(b + L.sx[ks]);
  st.sy = (const C2<T>*)(b + L.sy[ks]);
  st.sz = (const C2<T>*)(b + L.sz[ks]);
  st.xfac = (const T*)(b + L.xf);
  st.yfac = (const T*)(b + L.yf);
  st.zfac = (const T*)(b + L.zf);
  st.xdif = (const T*)(b + L.xd);
  st.ydif = (const T*)(b + L.yd);
  st.zdif = (const T*)(b + L.zd);
  st.forc = (c.p.kforce > 0) ? (const C2<T>*)c.d_forc : nullptr;
  st.kfor = c.kfor; st.k2fo = c.k2fo;
  st.kforce2 = c.p.kforce * c.p.kforce;
  st.b11 = (T)(c.p.beta1 * c.p.beta1);
  st.b22 = (T)(c.p.beta2 * c.p.beta2);
  st.b33 = (T)(c.p.beta3 * c.p.beta3);
  st.norm = (T)(c.dt2 / c.n / c.n);
  st.spf = (const T*)c.d_spf;
  return st;
}

// stage tables of both stages for the shifts in c.gsh (shifts.f:146-178)
template <typename T>
static void fill_shift_tables(Ctx& c) {
  TabLayout<T> L(c.n);
  char* b = (char*)c.h_tabs;
  const int n = c.n;
  const double pi = 4. * std::atan(1.);
  const double ph = 2. * pi / n;
  for (int k = 0; k < 2; k++) {
    C2<T>* sx = (C2<T>*)(b + L.sx[k]);
    C2<T>* sy = (C2<T>*)(b + L.sy[k]);
    C2<T>* sz = (C2<T>*)(b + L.sz[k]);
    for (int x = 0; x <= n / 2; x++) {
      const double th = (ph * c.g.kx[x]) * c.gsh[0][k];
      sx[x] = cmk<C2<T>>((T)std::cos(th), (T)std::sin(th));
    }
    for (int y = 0; y < n; y++) {
      const double th = (ph * c.g.ky[y]) * c.gsh[1][k];
      sy[y] = cmk<C2<T>>((T)std::cos(th), (T)std::sin(th));
    }
    for (int z = 0; z < n; z++) {
      const double th = (ph * c.g.kz[z]) * c.gsh[2][k];
      sz[z] = cmk<C2<T>>((T)std::cos(th), (T)std::sin(th));
    }
  }
}

static int upload_tables(Ctx& c) {
  const size_t tot = c.prec == PSDNS_PREC_FP64 ? TabLayout<double>(c.n).total : TabLayout<float>(c.n).total;
  CK(cudaMemcpyAsync(c.d_tabs, c.h_tabs, tot, cudaMemcpyHostToDevice, c.stream));
  // the staging buffer is reused by the next fill: wait for the copy
  CK(cudaStreamSynchronize(c.stream));
  return 0;
}


// ---------------------------------------------------------------------------
// per-(precision, n, nc) kernel launch sequence
// ---------------------------------------------------------------------------
template <typename T, int N, int NC> struct Impl {
  using C = C2<T>;
  using TL = Tiles<T>;
  static constexpr int L = LS<N>::value;
  static constexpr size_t TWB = sizeof(C) * FFTPlan<T, N>::TWSIZE;
  static size_t sm1() { return TWB + sizeof(C) * TL::TB_I * L; }
  static size_t sm2() { return TWB + sizeof(C) * TL::XT2 * L; }
  static size_t sm3() { return K3Launch<T, N, NC>::SMEM; }
  static size_t sm4() { return K4Launch<T, N>::SMEM; }
  static size_t sm5() { return TWB + sizeof(C) * (4 + NC) * TL::TB_F * L; }
  static size_t sm2tc() { return TWB + sizeof(C) * kTcXT2 * L + kTcTail; }
  static size_t sm4tc() { return K4LaunchX<T, N, kTcXT4, true>::SMEM + kTcTail; }

  // the tensor-core form (FP32 state at n = 1024): the same kernels with
  // their 1-D transforms on the tensor cores, and a shared-memory tail
  static constexpr bool kTc = std::is_same<T, float>::value && N == 1024;
  static TcArgs tc_args(const Ctx& c) { return TcArgs{(const uint4*)c.d_tcb, c.d_tw2, c.d_tcerr}; }

  static int setup() {
    if constexpr (kTc) {
      CK(cudaFuncSetAttribute(k_yinv<T, N, false, NC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sm1() + kTcTail)));
      CK(cudaFuncSetAttribute(k_zinv<T, N, NC, false, true, kTcXT2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sm2tc()));
      CK(cudaFuncSetAttribute(k_xchain<T, N, NC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)K3Launch<T, N, NC>::SMEM_TC));
      CK(cudaFuncSetAttribute(k_zfwd<T, N, NC, true, kTcXT4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sm4tc()));
      CK(cudaFuncSetAttribute(k_yfwd<T, N, 1, NC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sm5() + kTcTail)));
      CK(cudaFuncSetAttribute(k_yfwd<T, N, 2, NC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sm5() + kTcTail)));
    }
    CK(cudaFuncSetAttribute(k_yinv<T, N, false, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1()));
    CK(cudaFuncSetAttribute(k_zinv<T, N, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2()));
    CK(cudaFuncSetAttribute(k_xchain<T, N, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm3()));
    CK(cudaFuncSetAttribute(k_zfwd<T, N, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm4()));
    CK(cudaFuncSetAttribute(k_yfwd<T, N, 1, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm5()));
    if constexpr (NC == 0) {
      CK(cudaFuncSetAttribute(k_yfwd<T, N, 11>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm5()));
      CK(cudaFuncSetAttribute(k_yfwd<T, N, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm5()));
      CK(cudaFuncSetAttribute(k_yfwd<T, N, 13>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm5()));
      CK(cudaFuncSetAttribute(k_yfwd<T, N, 14>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm5()));
    }
    CK(cudaFuncSetAttribute(k_yfwd<T, N, 2, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm5()));
    CK(cudaFuncSetAttribute(k_zinv<T, N, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2()));
    CK(cudaFuncSetAttribute(k_yfwd<T, N, 0, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(sm5() + sizeof(double) * (N / 2))));
    CK(cudaFuncSetAttribute(k_xmoments<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)KMomLaunch<T, N>::SMEM));
    // the particle path transforms the velocity only (NC = 0 instances)
    CK(cudaFuncSetAttribute(k_zinv<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2()));
    CK(cudaFuncSetAttribute(k_yinv<T, N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1()));
    CK(cudaFuncSetAttribute(k_xspline<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smxs()));
    return 0;
  }

  static size_t smxs() { return TWB + sizeof(C) * 3 * (TL::TZ / 2) * L; }

  // particles at stage 1 (lagpart.f -> partsp.f): spline coefficients of the
  // stage-1 field on the predictor grid, then the particle RK2 step with the
  // previous step's dt (realspace is called before step, timestep_module.f)
  static int particles(Ctx& c) {
    Geo g = make_geo(c);
    StageTables<T> st = make_tables<T>(c, 0);
    const C* tw = (const C*)c.d_tw;
    C* ub = (C*)c.d_ub;
    C* uz = (C*)c.d_uz;
    const int kxn = c.g.kxn;
    prof_mark(c, 0, 5, 0);
    k_yinv<T, N, true><<<dim3(k1_blocks<T>(c.nab_i), 3), K1Launch<T, N>::THREADS, sm1(), c.stream>>>(g, st, (const C*)c.d_u,
                                                                                               ub, tw);
    k_zinv<T, N><<<dim3(N, (kxn + TL::XT2 - 1) / TL::XT2, 3), Launch<T, N, TL::XT2>::THREADS, sm2(), c.stream>>>(
        g, ub, uz, tw);
    using V4 = typename V4T<T>::type;
    k_xspline<T, N><<<dim3(c.nzt, N), Launch<T, N, 2 * TL::TZ>::THREADS, smxs(), c.stream>>>(g, uz, (V4*)c.d_bs, tw);
    const double pi = 4. * std::atan(1.);
    const double ps = 1.0;
    const double fact = ((((0.5 * c.dt) / 2.) / pi) * (double)N) * ps;   // rk_advpos.f:31-32
    const long long groups = (c.np + 15) / 16;
    const int blocks = (int)std::min<long long>((groups + 15) / 16, 148LL * 16);
    k_particles<T><<<blocks, 256, 0, c.stream>>>((const V4*)c.d_bs, N, c.np, c.d_pos, c.d_vel, c.gsh[0][0],
                                                 c.gsh[1][0], c.gsh[2][0], fact, fact, c.part_first ? 1 : 0);
    prof_mark(c, 0, 5, 1);
    CK(cudaGetLastError());
    c.part_first = false;
    return 0;
  }

  // vgmomt.f: moments 1..8 of du/dx and dw/dz of u or un on the grid
  // shifted by gsh (written as the stage-1 shifts for the duration)
  static int moments(Ctx& c, int which, const double* gsh, double* out) {
    double save[3][2];
    std::memcpy(save, c.gsh, sizeof save);
    for (int i = 0; i < 3; i++) c.gsh[i][0] = gsh ? gsh[i] : 0.0;
    fill_shift_tables<T>(c);
    int rc = upload_tables(c);
    std::memcpy(c.gsh, save, sizeof save);
    if (rc) return 1;
    Geo g = make_geo(c);
    StageTables<T> st = make_tables<T>(c, 0);
    const C* tw = (const C*)c.d_tw;
    C* ub = (C*)c.d_ub;
    C* uz = (C*)c.d_uz;
    const int kxn = c.g.kxn;
    k_yinv<T, N><<<dim3(c.nab_i, 3), K1Launch<T, N>::THREADS, sm1(), c.stream>>>(
        g, st, (const C*)(which == PSDNS_FIELD_U ? c.d_u : c.d_un), ub, tw);
    k_zinv<T, N, 0, true><<<dim3(N, (kxn + TL::XT2 - 1) / TL::XT2, 2), Launch<T, N, TL::XT2>::THREADS, sm2(),
                           c.stream>>>(g, ub, uz, tw, st.b11, st.b33);
    // the transposed copy in ub is consumed: its space holds the partial sums
    double* partial = (double*)c.d_ub;
    double* d_out = partial + (size_t)c.nzt * N * 16;
    k_xmoments<T, N><<<dim3(c.nzt, N), KMomLaunch<T, N>::THREADS, KMomLaunch<T, N>::SMEM, c.stream>>>(g, uz, tw,
                                                                                                    partial);
    k_moments_reduce<<<16, 256, 0, c.stream>>>(partial, (long long)c.nzt * N, 1.0 / ((double)N * N * N), d_out);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d_out, 16 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    // the next step refills its tables from c.gsh; restore the uploaded ones too
    fill_shift_tables<T>(c);
    return upload_tables(c);
  }

  // trfsp.f: transfer spectrum T(k) = sum over shell k of tfact
  // Re(conj(un) . N(u)), N the convective term of a stage-1 evaluation on the
  // grid shifted by gsh (stage-1 shifts of the step; null = unshifted).  The
  // reference divides w = (dt/2) N by dt/2 (fmult = 2/dt); here the stage
  // runs with dt/2 = 1.
  static int transfer(Ctx& c, const double* gsh, double* tk) {
    double save[3][2];
    std::memcpy(save, c.gsh, sizeof save);
    const double dt2 = c.dt2;
    for (int i = 0; i < 3; i++) c.gsh[i][0] = gsh ? gsh[i] : 0.0;
    fill_shift_tables<T>(c);
    int rc = upload_tables(c);
    std::memcpy(c.gsh, save, sizeof save);
    if (rc) return 1;
    c.dt2 = 1.0;
    rc = stage_a(c, 1);
    if (!rc) {
      Geo g = make_geo(c);
      StageTables<T> st = make_tables<T>(c, 0);
      st.tdk = std::min(c.p.beta1, std::min(c.p.beta2, c.p.beta3));
      double* d_tk = (double*)c.d_efkz;   // n/2 + 2 shells of 3 doubles: room for n/2
      if (cudaMemsetAsync(d_tk, 0, sizeof(double) * (N / 2), c.stream) != cudaSuccess) rc = set_error("memset");
      if (!rc) {
        k_yfwd<T, N, 0, NC><<<c.nab_f, K5Launch<T, N, NC>::THREADS, sm5() + sizeof(double) * (N / 2), c.stream>>>(
            g, st, (const C*)c.d_ub, (C*)c.d_u, (C*)c.d_un, (const C*)c.d_tw, d_tk);
        if (cudaGetLastError() != cudaSuccess) rc = set_error("transfer launch failed");
      }
      if (!rc && (cudaMemcpyAsync(tk, d_tk, sizeof(double) * (N / 2), cudaMemcpyDeviceToHost, c.stream) !=
                      cudaSuccess ||
                  cudaStreamSynchronize(c.stream) != cudaSuccess))
        rc = set_error("transfer copy failed");
      // efkz is zeroed again by the next forced stage 1
      if (!rc && cudaMemsetAsync(d_tk, 0, sizeof(double) * (N / 2), c.stream) != cudaSuccess) rc = set_error("memset");
    }
    c.dt2 = dt2;
    fill_shift_tables<T>(c);
    if (upload_tables(c)) return 1;
    return rc;
  }

  static int twiddles(Ctx& c) {
    std::vector<C> tw(FFTPlan<T, N>::TWSIZE);
    build_twiddles<T, N>(tw.data());
    CK(cudaMalloc(&c.d_tw, sizeof(C) * tw.size()));
    CK(cudaMemcpy(c.d_tw, tw.data(), sizeof(C) * tw.size(), cudaMemcpyHostToDevice));
    return 0;
  }

  // stage part A: K1..K4 (through the forward z transform)
  static int stage_a(Ctx& c, int kstep) {
    if constexpr (kTc)
      if (c.dft == PSDNS_DFT_TC_BF16X3) return stage_a_tc(c, kstep);
    Geo g = make_geo(c);
    StageTables<T> st = make_tables<T>(c, (kstep - 1) & 1);
    const C* tw = (const C*)c.d_tw;
    C* u = (C*)c.d_u;
    C* ub = (C*)c.d_ub;
    C* uz = (C*)c.d_uz;
    const int kxn = c.g.kxn;
    const int s = kstep - 1;
    {
      constexpr int TH = K1Launch<T, N>::THREADS;
      prof_mark(c, s, 0, 0);
      k_yinv<T, N, false, NC><<<dim3(k1_blocks<T>(c.nab_i), 3 + 2 * NC), TH, sm1(), c.stream>>>(g, st, u, ub, tw);
      prof_mark(c, s, 0, 1);
    }
    {
      constexpr int TH = Launch<T, N, TL::XT2>::THREADS;
      prof_mark(c, s, 1, 0);
      k_zinv<T, N, NC><<<dim3(N, (kxn + TL::XT2 - 1) / TL::XT2, 3 + 3 * NC), TH, sm2(), c.stream>>>(
          g, ub, uz, tw, st.b11, st.b33);
      prof_mark(c, s, 1, 1);
    }
    {
      constexpr int TH = K3Launch<T, N, NC>::THREADS;
      prof_mark(c, s, 2, 0);
      // mean-gradient coefficients cb = beta * grad (init.f:42-45)
      const T cb1 = (T)(c.p.beta1 * c.p.grad[0]), cb2 = (T)(c.p.beta2 * c.p.grad[1]),
              cb3 = (T)(c.p.beta3 * c.p.grad[2]);
      k_xchain<T, N, NC><<<dim3(c.nzt, N), TH, sm3(), c.stream>>>(g, uz, tw, st.b11, st.b22, st.b33, c.d_velmax,
                                                                    kstep == 1 ? 1 : 0, cb1, cb2, cb3);
      prof_mark(c, s, 2, 1);
    }
    {
      constexpr int TH = K4Launch<T, N>::THREADS;
      prof_mark(c, s, 3, 0);
      constexpr int XT4 = k4_xt(sizeof(T) == 8, N);
      k_zfwd<T, N, NC><<<dim3(N / TL::YT4, (kxn + XT4 - 1) / XT4), TH, sm4(), c.stream>>>(g, uz, ub, tw,
                                                                                                   st.b11, st.b33);
      prof_mark(c, s, 3, 1);
    }
    CK(cudaGetLastError());
    return 0;
  }

  // stage part A with the 1-D transforms on the tensor cores (same launch
  // grids as stage_a)
  static int stage_a_tc(Ctx& c, int kstep) {
    Geo g = make_geo(c);
    StageTables<T> st = make_tables<T>(c, (kstep - 1) & 1);
    const TcArgs ta = tc_args(c);
    const C* tw = (const C*)c.d_tw;
    C* u = (C*)c.d_u;
    C* ub = (C*)c.d_ub;
    C* uz = (C*)c.d_uz;
    const int kxn = c.g.kxn;
    const int s = kstep - 1;
    prof_mark(c, s, 0, 0);
    k_yinv<T, N, false, NC, true><<<dim3(k1_blocks<T>(c.nab_i), 3 + 2 * NC), K1Launch<T, N>::THREADS,
                                    sm1() + kTcTail, c.stream>>>(g, st, u, ub, tw, ta);
    prof_mark(c, s, 0, 1);
    prof_mark(c, s, 1, 0);
    k_zinv<T, N, NC, false, true, kTcXT2><<<dim3(N, (kxn + kTcXT2 - 1) / kTcXT2, 3 + 3 * NC),
                                            Launch<T, N, kTcXT2>::THREADS, sm2tc(), c.stream>>>(
        g, ub, uz, tw, st.b11, st.b33, ta);
    prof_mark(c, s, 1, 1);
    prof_mark(c, s, 2, 0);
    const T cb1 = (T)(c.p.beta1 * c.p.grad[0]), cb2 = (T)(c.p.beta2 * c.p.grad[1]),
            cb3 = (T)(c.p.beta3 * c.p.grad[2]);
    k_xchain<T, N, NC, true><<<dim3(c.nzt, N), K3Launch<T, N, NC>::THREADS, K3Launch<T, N, NC>::SMEM_TC,
                               c.stream>>>(g, uz, tw, st.b11, st.b22, st.b33, c.d_velmax, kstep == 1 ? 1 : 0, cb1,
                                           cb2, cb3, ta);
    prof_mark(c, s, 2, 1);
    prof_mark(c, s, 3, 0);
    k_zfwd<T, N, NC, true, kTcXT4><<<dim3(N / TL::YT4, (kxn + kTcXT4 - 1) / kTcXT4),
                                     K4LaunchX<T, N, kTcXT4, true>::THREADS, sm4tc(), c.stream>>>(g, uz, ub, tw, st.b11,
                                                                                          st.b33, ta);
    prof_mark(c, s, 3, 1);
    CK(cudaGetLastError());
    return 0;
  }

  static int stage_b_tc(Ctx& c, int kstep) {
    Geo g = make_geo(c);
    StageTables<T> st = make_tables<T>(c, (kstep - 1) & 1);
    const TcArgs ta = tc_args(c);
    constexpr int TH = K5Launch<T, N, NC>::THREADS;
    prof_mark(c, kstep - 1, 4, 0);
    if (kstep == 1)
      k_yfwd<T, N, 1, NC, true><<<c.nab_f, TH, sm5() + kTcTail, c.stream>>>(
          g, st, (const C*)c.d_ub, (C*)c.d_u, (C*)c.d_un, (const C*)c.d_tw, c.d_efkz, ta);
    else
      k_yfwd<T, N, 2, NC, true><<<c.nab_f, TH, sm5() + kTcTail, c.stream>>>(
          g, st, (const C*)c.d_ub, (C*)c.d_u, (C*)c.d_un, (const C*)c.d_tw, c.d_efkz, ta);
    prof_mark(c, kstep - 1, 4, 1);
    CK(cudaGetLastError());
    return 0;
  }

  // stage part B: K5
  // K5 of the RK4 sub-stages (velocity only)
  static int stage_b_rk4(Ctx& c, int kstep) {
    if constexpr (NC == 0) {
      Geo g = make_geo(c);
      StageTables<T> st = make_tables<T>(c, (kstep - 1) & 1);
      constexpr int TH = K5Launch<T, N, NC>::THREADS;
      const C* ub = (const C*)c.d_ub;
      C *u = (C*)c.d_u, *un = (C*)c.d_un, *r = (C*)c.d_u1;
      const C* tw = (const C*)c.d_tw;
      prof_mark(c, kstep - 1, 4, 0);
      switch (kstep) {
        case 1: k_yfwd<T, N, 11><<<c.nab_f, TH, sm5(), c.stream>>>(g, st, ub, u, un, tw, c.d_efkz, TcArgs(), r); break;
        case 2: k_yfwd<T, N, 12><<<c.nab_f, TH, sm5(), c.stream>>>(g, st, ub, u, un, tw, c.d_efkz, TcArgs(), r); break;
        case 3: k_yfwd<T, N, 13><<<c.nab_f, TH, sm5(), c.stream>>>(g, st, ub, u, un, tw, c.d_efkz, TcArgs(), r); break;
        default: k_yfwd<T, N, 14><<<c.nab_f, TH, sm5(), c.stream>>>(g, st, ub, u, un, tw, c.d_efkz, TcArgs(), r);
      }
      prof_mark(c, kstep - 1, 4, 1);
      CK(cudaGetLastError());
      return 0;
    } else {
      return set_error("RK4 advances the velocity only (nc = 0)");
    }
  }

  static int stage_b(Ctx& c, int kstep) {
    if (c.rk == 4) return stage_b_rk4(c, kstep);
    if constexpr (kTc)
      if (c.dft == PSDNS_DFT_TC_BF16X3) return stage_b_tc(c, kstep);
    Geo g = make_geo(c);
    StageTables<T> st = make_tables<T>(c, (kstep - 1) & 1);
    constexpr int TH = K5Launch<T, N, NC>::THREADS;
    prof_mark(c, kstep - 1, 4, 0);
    if (kstep == 1)
      k_yfwd<T, N, 1, NC><<<c.nab_f, TH, sm5(), c.stream>>>(g, st, (const C*)c.d_ub, (C*)c.d_u, (C*)c.d_un,
                                                        (const C*)c.d_tw, c.d_efkz);
    else
      k_yfwd<T, N, 2, NC><<<c.nab_f, TH, sm5(), c.stream>>>(g, st, (const C*)c.d_ub, (C*)c.d_u, (C*)c.d_un,
                                                        (const C*)c.d_tw, c.d_efkz);
    prof_mark(c, kstep - 1, 4, 1);
    CK(cudaGetLastError());
    return 0;
  }
};

struct Ops {
  int (*setup)();
  int (*twiddles)(Ctx&);
  int (*stage_a)(Ctx&, int);
  int (*stage_b)(Ctx&, int);
  int (*particles)(Ctx&);
  int (*moments)(Ctx&, int, const double*, double*);
  int (*transfer)(Ctx&, const double*, double*);
};

template <typename T, int N, int NC> Ops ops_for() {
  using I = Impl<T, N, NC>;
  return Ops{&I::setup, &I::twiddles, &I::stage_a, &I::stage_b, &I::particles, &I::moments, &I::transfer};
}

template <int N> Ops ops_n(int prec, int nc) {
  if (prec == PSDNS_PREC_FP64) return nc ? ops_for<double, N, 1>() : ops_for<double, N, 0>();
  return nc ? ops_for<float, N, 1>() : ops_for<float, N, 0>();
}

}  // namespace psdns
#include "ensemble_impl.cuh"
namespace psdns {

// The kernels of each grid size are instantiated in a unit of their own
// (this file compiled with -DPSDNS_INST_N=n), so that the library builds in
// parallel; the main unit (no PSDNS_INST_N) holds the host code.
#define PSDNS_FOR_EACH_N(X) X(16) X(32) X(48) X(64) X(96) X(128) X(256) X(512) X(1024)
#ifdef PSDNS_INST_N
template Ops ops_n<PSDNS_INST_N>(int, int);
template int ens_setup_n<PSDNS_INST_N>(EnsClass&);
}  // namespace psdns
#else
#define PSDNS_EXTERN_N(NN) extern template Ops ops_n<NN>(int, int); extern template int ens_setup_n<NN>(EnsClass&);
PSDNS_FOR_EACH_N(PSDNS_EXTERN_N)
#undef PSDNS_EXTERN_N

static bool get_ops(int prec, int n, int nc, Ops& o) {
#define PSDNS_CASE(NN)    \
  case NN:                \
    o = ops_n<NN>(prec, nc); \
    return true;
  switch (n) {
    PSDNS_CASE(16)
    PSDNS_CASE(32)
    PSDNS_CASE(48)
    PSDNS_CASE(64)
    PSDNS_CASE(96)
    PSDNS_CASE(128)
    PSDNS_CASE(256)
    PSDNS_CASE(512)
    PSDNS_CASE(1024)
    default:
      return false;
  }
#undef PSDNS_CASE
}

// ---------------------------------------------------------------------------
// shifts (PSDNS/shifts.f:40-178, compiled with -DRKFOUR as in the makefile,
// which draws gsh(:,3:4) as well) and stage tables
// ---------------------------------------------------------------------------
static double cancel(double d) { return std::fmod(d + 0.5, 1.); }

static void draw_shifts(Ctx& c) {
  const int ks = c.p.kshift;
  if (c.istart <= 0 && c.jstep == 1 && (ks == 1 || ks == 3)) {
    c.rng.ranseq(c.p.ksran);
    for (int i = 0; i < 3; i++) c.gsh[i][1] = c.rng.ranu();
    for (int i = 0; i < 3; i++) c.gsh4[i][1] = c.rng.ranu();
  }
  if (ks == 1 || ks == 2) c.rng.ranseq(c.p.ksran);
  for (int pass = 0; pass < 2; pass++) {
    double(*g)[2] = pass == 0 ? c.gsh : c.gsh4;
    for (int i = 0; i < 3; i++) {
      if (ks == 1) { g[i][0] = cancel(g[i][1]); g[i][1] = c.rng.ranu(); }
      else if (ks == 2) { g[i][0] = c.rng.ranu(); g[i][1] = cancel(g[i][0]); }
      else if (ks == 3) { g[i][0] = cancel(g[i][1]); g[i][1] = cancel(g[i][0]); }
      else { g[i][0] = 0.; g[i][1] = 0.; }
    }
  }
}

template <typename T>
static void fill_factor_tables(Ctx& c) {
  TabLayout<T> L(c.n);
  char* b = (char*)c.h_tabs;
  const int n = c.n;
  T* xf = (T*)(b + L.xf);
  T* yf = (T*)(b + L.yf);
  T* zf = (T*)(b + L.zf);
  const double b11 = c.p.beta1 * c.p.beta1, b22 = c.p.beta2 * c.p.beta2, b33 = c.p.beta3 * c.p.beta3;
  const double nu = c.p.viscos;
  double term = b11 * c.dt;
  for (int x = 0; x <= n / 2; x++) xf[x] = (T)std::exp(-(nu * (c.g.kx[x] * c.g.kx[x]) * term));
  term = b22 * c.dt;
  for (int y = 0; y < n; y++) yf[y] = (T)std::exp(-(nu * (c.g.ky[y] * c.g.ky[y]) * term));
  term = b33 * c.dt;
  for (int z = 0; z < n; z++) zf[z] = (T)std::exp(-(nu * (c.g.kz[z] * c.g.kz[z]) * term));
  if (c.nc > 0) {
    // scalar factors xfac**(1/pr) from the FP64 velocity factors (step.f:387-407)
    T* xd = (T*)(b + L.xd);
    T* yd = (T*)(b + L.yd);
    T* zd = (T*)(b + L.zd);
    const double ipr = 1. / c.p.pr;
    term = b11 * c.dt;
    for (int x = 0; x <= n / 2; x++) xd[x] = (T)std::pow(std::exp(-(nu * (c.g.kx[x] * c.g.kx[x]) * term)), ipr);
    term = b22 * c.dt;
    for (int y = 0; y < n; y++) yd[y] = (T)std::pow(std::exp(-(nu * (c.g.ky[y] * c.g.ky[y]) * term)), ipr);
    term = b33 * c.dt;
    for (int z = 0; z < n; z++) zd[z] = (T)std::pow(std::exp(-(nu * (c.g.kz[z] * c.g.kz[z]) * term)), ipr);
  }
}

// step.f:49-99, :247-262, :280-295.  Returns nonzero on the reference's abort
// conditions (the step is still completed; the caller decides).
static int step_control(Ctx& c) {
  c.dt = c.dt0;
  int err = 0;
  if (c.p.cfl > 0.) {
    c.dt = c.p.cfl / c.velmax;
    if (c.velmax < .001) err = set_error("velmax %.6e below 0.001 (step.f:79)", c.velmax);
  }
  c.time = c.time + c.dt;
  if (c.dt == 0.) err = set_error("dt unexpectedly zero (step.f:256)");
  c.dt2 = c.dt / 2.;
  if (c.p.cfl > 0.) {
    if (c.dt > 10. || c.dt < 1.e-7) err = set_error("dt out of control: %.6e (step.f:280)", c.dt);
  } else if (c.p.cfl < 0.) {
    const double cn = c.velmax * c.dt / 2. / (4. * std::atan(1.));
    if (cn > 1) err = set_error("courant number %.4f exceeds 1 (step.f:292)", cn);
  }
  return err;
}

// for(kfor,k2fo,k2fo,3) complex double -> device precision -> d_forc
static int upload_forcing(Ctx& c, const double* tab) {
  const size_t nf = (size_t)c.kfor * c.k2fo * c.k2fo * 3;
  if (c.prec == PSDNS_PREC_FP64) {
    std::memcpy(c.h_forc, tab, nf * sizeof(double2));
  } else {
    float2* f = (float2*)c.h_forc;
    for (size_t i = 0; i < nf; i++) f[i] = make_float2((float)tab[2 * i], (float)tab[2 * i + 1]);
  }
  CK(cudaMemcpyAsync(c.d_forc, c.h_forc, nf * c.csz, cudaMemcpyHostToDevice, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return 0;
}

// forcdt.f:18-41: energy input per shell from efkz (device, FP64)
static int collect_forcing_stats(Ctx& c) {
  if (!(c.p.kforce > 0)) return 0;
  std::vector<double> e(3 * (c.n / 2 + 2));
  CK(cudaMemcpyAsync(e.data(), c.d_efkz, sizeof(double) * e.size(), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  c.efk_host.assign(c.kfor, 0.0);
  c.erate = 0;
  c.eirate[0] = c.eirate[1] = c.eirate[2] = 0;
  for (int k = 0; k < c.kfor; k++) {
    const double e1 = e[3 * k] / c.dt, e2 = e[3 * k + 1] / c.dt, e3 = e[3 * k + 2] / c.dt;
    c.efk_host[k] = .5 * (e1 + e2 + e3);
    c.eirate[0] += e1; c.eirate[1] += e2; c.eirate[2] += e3;
    c.erate += c.efk_host[k];
  }
  return 0;
}

// hooks/LAG_LOCAL/partin.f:93-131 (pstart = 0: nop uniform random positions,
// nearly equal numbers per y-slice, from RNG sequence kipran; ranu2.f with
// RANDOM_SEED shares the seed of ranu) and :141-190 (pstart = -1: a cubic
// lattice of nop^3 grid nodes).  Grid planes gx(i) = 1 + (i-1)/beta1 +
// gsh(1,1) (partsp.f:44-53) with this step's stage-1 shifts.
static int make_partin(Ctx& c) {
  const int n = c.n;
  const double ps1 = std::sqrt(c.p.beta1 * c.p.beta1), ps2 = std::sqrt(c.p.beta2 * c.p.beta2),
               ps3 = std::sqrt(c.p.beta3 * c.p.beta3);
  long long nop = c.pin_pstart == -1 ? c.pin_nop * c.pin_nop * c.pin_nop : c.pin_nop;
  std::vector<double> pos(3 * (size_t)nop);
  if (c.pin_pstart == 0) {
    const double gx1 = 1. + 0. / ps1 + c.gsh[0][0], gz1 = 1. + 0. / ps3 + c.gsh[2][0];
    const long long npy = nop / n, npe = nop - npy * n;
    long long niny = 0;
    c.rng.ranseq(c.pin_kipran);
    for (int y = 1; y <= n; y++) {
      const long long ni = npy + (y <= npe ? 1 : 0);
      for (int k = 0; k < 3; k++)
        for (long long i = 0; i < ni; i++) pos[k * nop + niny + i] = c.rng.ranu();
      const double gy = 1. + (double)(y - 1) / ps2 + c.gsh[1][0];
      for (long long i = 0; i < ni; i++) {
        const long long m = niny + i;
        pos[m] = pos[m] * (double)n + gx1;
        pos[nop + m] = pos[nop + m] / ps2 + gy;
        pos[2 * nop + m] = pos[2 * nop + m] * (double)n + gz1;
      }
      niny += ni;
    }
  } else {
    const long long npu = c.pin_nop;
    long long it[3], i1[3], i2[3];
    for (int d = 0; d < 3; d++) {
      it[d] = n / npu + (n % npu ? 1 : 0);
      i1[d] = std::max(1LL, n / 2 + 1 - npu / 2 * it[d] + it[d] / 2);
      i2[d] = std::min((long long)n, n / 2 + 1 + npu / 2 * it[d] - it[d] / 2);
    }
    const double psv[3] = {ps1, ps2, ps3};
    long long idx = 0;
    for (long long k = i1[2]; k <= i2[2]; k += it[2])
      for (long long j = i1[1]; j <= i2[1]; j += it[1])
        for (long long i = i1[0]; i <= i2[0]; i += it[0]) {
          if (idx < nop) {
            pos[idx] = 1. + (double)(i - 1) / psv[0] + c.gsh[0][0];
            pos[nop + idx] = 1. + (double)(j - 1) / psv[1] + c.gsh[1][0];
            pos[2 * nop + idx] = 1. + (double)(k - 1) / psv[2] + c.gsh[2][0];
          }
          idx++;
        }
    if (idx != nop) return set_error("partin: the lattice has %lld nodes, not %lld (partin.f:129)", idx, nop);
  }
  c.pin_nop = 0;
  if (psdns_gpu_particles_set(&c, nop, pos.data())) return 1;
  return 0;
}

static int run_stage(Ctx& c, const Ops& o, int kstep, int* ctl_err) {
  if (kstep == 1 && c.pin_nop > 0 && make_partin(c)) return 1;
  if (kstep == 1 && c.np > 0 && o.particles(c)) return 1;
  if (kstep == 1) CK(cudaMemsetAsync(c.d_velmax, 0, sizeof(unsigned long long), c.stream));
  if (o.stage_a(c, kstep)) return 1;
  if (kstep == 1) {
    CK(cudaMemcpyAsync(c.h_velmax, c.d_velmax, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    prof_collect(c, 0, 0, 4);
    if (c.np > 0) prof_collect(c, 0, 5, 6);
    double vm;
    std::memcpy(&vm, c.h_velmax, sizeof vm);
    c.velmax = vm;
    if (c.d_tcerr) {
      unsigned e = 0;
      CK(cudaMemcpy(&e, c.d_tcerr, sizeof e, cudaMemcpyDeviceToHost));
      if (e) return set_error("a tensor-core transform gave up waiting for its MMAs (error word %u)", e);
    }
    *ctl_err = step_control(c);
    if (c.prec == PSDNS_PREC_FP64) fill_factor_tables<double>(c); else fill_factor_tables<float>(c);
    if (upload_tables(c)) return 1;
    if (c.p.kforce > 0) {
      // force.f, called after step at stage 1 (timestep_module.f:261-263)
      c.forcing.step(c.rng, c.dt, c.istart);
      if (upload_forcing(c, c.forcing.table.data())) return 1;
      CK(cudaMemsetAsync(c.d_efkz, 0, sizeof(double) * 3 * (c.n / 2 + 2), c.stream));
    }
  }
  if (o.stage_b(c, kstep)) return 1;
  return 0;
}

// sptr.f:139-193 shell sums on the device (FP64), :235-237 and :350-400 on
// the host, for the state at src (one box, geometry g); scratch holds
// n * kSpecVals doubles
static int spectra_of(const Geo& g, const void* src, int prec, const psdns_params& p, cudaStream_t stream,
                      void* scratch, double* ek, double* dk, double* eijk, double* stats) {
  const int n = g.n, ns = n;   // mxyz = max(nx,ny,nz)/beta_min shells (comsp_set.f:14)
  const size_t nv = (size_t)ns * kSpecVals;
  double* d_out = (double*)scratch;
  CK(cudaMemsetAsync(d_out, 0, nv * sizeof(double), stream));
  const double b11 = p.beta1 * p.beta1, b22 = p.beta2 * p.beta2, b33 = p.beta3 * p.beta3;
  const size_t smem = nv * sizeof(double);
  if (prec == PSDNS_PREC_FP64) {
    CK(cudaFuncSetAttribute(k_spectra<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_spectra<double><<<148 * 2, 512, smem, stream>>>(g, (const double2*)src, b11, b22, b33, ns, d_out);
  } else {
    CK(cudaFuncSetAttribute(k_spectra<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_spectra<float><<<148 * 2, 512, smem, stream>>>(g, (const float2*)src, b11, b22, b33, ns, d_out);
  }
  CK(cudaGetLastError());
  std::vector<double> h(nv);
  CK(cudaMemcpyAsync(h.data(), d_out, nv * sizeof(double), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  const double nu = p.viscos;
  double tke = 0, eps = 0, skew = 0, ekl = 0;
  for (int k = 0; k < ns; k++) {
    const double* v = &h[(size_t)k * kSpecVals];
    double e = 0.5 * (v[0] + v[3] + v[5]);
    double d = 0.5 * (2 * nu * v[6]);
    const double sk = 0.5 * (2 * nu * v[7]);
    if (k == 0) { e = 0; d = 0; }
    if (ek) ek[k] = e;
    if (dk) dk[k] = d;
    if (eijk) for (int j = 0; j < 6; j++) eijk[(size_t)k * 6 + j] = v[j];
    tke += e;
    eps += d;
    skew += sk;
    if (k < n / 2) ekl += v[8] / 2.;
  }
  const double pi = 4. * std::atan(1.);
  double klen = 0, kvel = 0, ktime = 0;
  if (eps > 0) {
    skew = 2. / 35. * std::pow(15. * nu / eps, 1.5) * skew;
    klen = std::pow(nu * nu * nu / eps, .25);
    kvel = std::pow(nu * eps, .25);
    ktime = std::pow(nu / eps, .5);
  }
  ekl = 1.5 * pi / (2 * tke) * ekl;
  if (stats) {
    stats[0] = tke; stats[1] = eps; stats[2] = skew; stats[3] = klen; stats[4] = kvel; stats[5] = ktime;
    stats[6] = ekl;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Asynchronous state copies (YCYL): the state is cut into kChunks contiguous
// pieces; H2D and D2H run on their own streams through complex(8) staging,
// so that the copies of one call overlap the conversions, and the upload of
// a state overlaps the download of the previous one (PCIe is full duplex).
// A chunk of set_state_async whose host range is that of a pending
// get_state_async waits only for that chunk's download.
// ---------------------------------------------------------------------------
// Every entry point on a context calls touch first: a sphere download still
// reading the state on s_out is joined into the context stream before any
// other work, except by the sphere upload, which waits for it chunk by chunk.
static void touch(Ctx* c, bool sphere_upload = false) {
  if (!c) return;
  c->api_calls++;
  if (c->sphere_get_pending && !sphere_upload) {
    for (int k = 0; k < Ctx::kChunks; k++) cudaStreamWaitEvent(c->stream, c->ev_d2h[k], 0);
    c->sphere_get_pending = false;
  }
}

// copy streams and events; with staging, also the complex(8) staging
// buffers of the full-array copies (the sphere copies need none)
static int async_setup(Ctx& c, bool staging = true) {
  if (staging && !c.d_in_stage) {
    const size_t bytes = sizeof(double2) * c.st_elems;
    size_t freeb = 0, totb = 0;
    CK(cudaMemGetInfo(&freeb, &totb));
    if (2 * bytes + (size_t)256 * 1024 * 1024 > freeb)
      return set_error("asynchronous state copies need %.2f GB of staging, %.2f GB free", 2 * bytes / 1e9,
                       freeb / 1e9);
    CK(cudaMalloc(&c.d_in_stage, bytes));
    CK(cudaMalloc(&c.d_out_stage, bytes));
  }
  if (c.s_in) return 0;
  CK(cudaStreamCreateWithFlags(&c.s_in, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c.s_out, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&c.ev_ready, cudaEventDisableTiming));
  for (int k = 0; k < Ctx::kChunks; k++) {
    CK(cudaEventCreateWithFlags(&c.ev_h2d[k], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c.ev_conv_in[k], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c.ev_conv_out[k], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c.ev_d2h[k], cudaEventDisableTiming));
  }
  return 0;
}

static void chunk_range(const Ctx& c, int k, size_t& off, size_t& cnt) {
  const size_t tot = c.st_elems, per = (tot + Ctx::kChunks - 1) / Ctx::kChunks;
  off = std::min(tot, per * k);
  cnt = std::min(tot, off + per) - off;
}

// sptr.f:199-218, :311-346 and :351-468 for the velocity: the normalised
// one-dimensional spectra xr, yr, zr ([6][n/2+1], pairs 11,12,13,22,23,33),
// and stats[55] = corr[6], lijk[6][3] (integral scales), rms[3], raak[3]
// (integral-scale Reynolds numbers), ett[3] (eddy turnover times),
// tmij[3][3] (mean square derivative of u_i along direction a), grdiss,
// taak[3][3] (Taylor microscales taylor(i,j,j)), tmre[3] (Taylor Reynolds
// numbers).  scratch holds 3 * 6 * (n/2+1) + 6 doubles.
static int spectra_scales_of(const Geo& g, const void* src, int prec, const psdns_params& p, cudaStream_t stream,
                             void* scratch, double* xr_out, double* yr_out, double* zr_out, double* stats) {
  const int n = g.n, nh = n / 2 + 1, NP = kSpec1dPairs;
  const size_t nv = (size_t)3 * NP * nh + NP;
  double* d_out = (double*)scratch;
  CK(cudaMemsetAsync(d_out, 0, nv * sizeof(double), stream));
  const double b22 = p.beta2 * p.beta2;
  const size_t smem = nv * sizeof(double);
  if (prec == PSDNS_PREC_FP64) {
    CK(cudaFuncSetAttribute(k_spectra_1d<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_spectra_1d<double><<<148 * 2, 512, smem, stream>>>(g, (const double2*)src, b22, d_out);
  } else {
    CK(cudaFuncSetAttribute(k_spectra_1d<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_spectra_1d<float><<<148 * 2, 512, smem, stream>>>(g, (const float2*)src, b22, d_out);
  }
  CK(cudaGetLastError());
  std::vector<double> h(nv);
  CK(cudaMemcpyAsync(h.data(), d_out, nv * sizeof(double), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  double* xr = h.data();
  double* yr = xr + NP * nh;
  double* zr = yr + NP * nh;
  double* der2 = zr + NP * nh;
  const double sv[3] = {p.beta1, p.beta2, p.beta3};
  const double s23 = sv[1] * sv[2], s31 = sv[2] * sv[0], s12 = sv[0] * sv[1], size = sv[0] * sv[1] * sv[2];
  const int pi_[NP] = {0, 0, 0, 1, 1, 2}, pj_[NP] = {0, 1, 2, 1, 2, 2};
  for (int ij = 0; ij < NP; ij++) {
    const double factor = sv[pi_[ij]] * sv[pj_[ij]];
    der2[ij] = der2[ij] * factor;
    for (int k = 0; k < nh; k++) {
      xr[ij * nh + k] = factor * xr[ij * nh + k] / size;
      yr[ij * nh + k] = factor * yr[ij * nh + k] / size;
      zr[ij * nh + k] = factor * zr[ij * nh + k] / size;
    }
  }
  const double pi = 4. * std::atan(1.), nu = p.viscos;
  double corr[NP];
  for (int ij = 0; ij < NP; ij++) {
    for (int k = 0; k < nh; k++) {
      xr[ij * nh + k] = s23 * xr[ij * nh + k];
      yr[ij * nh + k] = s31 * yr[ij * nh + k];
      zr[ij * nh + k] = s12 * zr[ij * nh + k];
    }
    double ssum = xr[ij * nh];
    for (int x = 1; x < n / 2; x++) ssum = ssum + 2. * xr[ij * nh + x];
    corr[ij] = sv[0] * ssum;
  }
  double lijk[NP][3] = {};
  for (int ij = 0; ij < NP; ij++)
    if (corr[ij] != 0.) {
      lijk[ij][0] = pi * xr[ij * nh] / corr[ij];
      lijk[ij][1] = pi * yr[ij * nh] / corr[ij];
      lijk[ij][2] = pi * zr[ij * nh] / corr[ij];
    }
  const int kt[3] = {0, 3, 5};
  double rms[3], raak[3] = {0, 0, 0}, ett[3] = {0, 0, 0}, tmij[3][3], taak[3][3], tmre[3] = {0, 0, 0};
  for (int i = 0; i < 3; i++) rms[i] = std::sqrt(corr[kt[i]]);
  if (nu > 0.)
    for (int i = 0; i < 3; i++) raak[i] = lijk[kt[i]][i] * rms[i] / nu;
  for (int i = 0; i < 3; i++)
    if (rms[i] != 0) ett[i] = lijk[kt[i]][i] / rms[i];
  for (int i = 0; i < 3; i++) {
    double ssum = 0.;
    for (int x = 1; x < n / 2; x++) ssum = ssum + (double)x * (double)x * xr[kt[i] * nh + x];
    tmij[i][0] = 2. * sv[0] * sv[0] * sv[0] * ssum;
    tmij[i][1] = der2[kt[i]];
    ssum = 0.;
    for (int z = 1; z < n / 2; z++) ssum = ssum + (double)z * (double)z * zr[kt[i] * nh + z];
    tmij[i][2] = 2. * sv[2] * sv[2] * sv[2] * ssum;
  }
  double grdiss = tmij[0][0] + tmij[1][1] + tmij[2][2] + tmij[0][1] + tmij[1][0] + tmij[0][2] + tmij[2][0] +
                  tmij[1][2] + tmij[2][1];
  grdiss = grdiss * nu;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) taak[i][j] = tmij[j][j] != 0. ? std::sqrt(corr[kt[i]] / tmij[j][j]) : 0.;
  if (nu > 0.)
    for (int i = 0; i < 3; i++) tmre[i] = taak[i][i] * rms[i] / nu;
  if (xr_out) std::memcpy(xr_out, xr, sizeof(double) * NP * nh);
  if (yr_out) std::memcpy(yr_out, yr, sizeof(double) * NP * nh);
  if (zr_out) std::memcpy(zr_out, zr, sizeof(double) * NP * nh);
  if (stats) {
    double* o = stats;
    for (int ij = 0; ij < NP; ij++) *o++ = corr[ij];
    for (int ij = 0; ij < NP; ij++)
      for (int a = 0; a < 3; a++) *o++ = lijk[ij][a];
    for (int i = 0; i < 3; i++) *o++ = rms[i];
    for (int i = 0; i < 3; i++) *o++ = raak[i];
    for (int i = 0; i < 3; i++) *o++ = ett[i];
    for (int i = 0; i < 3; i++)
      for (int a = 0; a < 3; a++) *o++ = tmij[i][a];
    *o++ = grdiss;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) *o++ = taak[i][j];
    for (int i = 0; i < 3; i++) *o++ = tmre[i];
  }
  return 0;
}

// one variable v of the state <-> the full half-complex layout on the host
// (complex(8) u(nxh, ny, nz)), staged in uz
static int full_var_set(Ctx& c, int v, const double* host) {
  const size_t fs = full_elems(c), vs = (size_t)c.g.xz_tot * c.n;
  if (fs * sizeof(double2) > c.uz_elems * c.csz) return set_error("full-layout staging does not fit");
  const Geo g = make_geo(c);
  CK(cudaMemcpyAsync(c.d_uz, host, sizeof(double2) * fs, cudaMemcpyHostToDevice, c.stream));
  if (c.prec == PSDNS_PREC_FP64)
    k_full_to_cyl<double><<<148 * 8, 256, 0, c.stream>>>(g, (const double2*)c.d_uz, (double2*)c.d_un + v * vs,
                                                           (double2*)c.d_u + v * vs);
  else
    k_full_to_cyl<float><<<148 * 8, 256, 0, c.stream>>>(g, (const double2*)c.d_uz, (float2*)c.d_un + v * vs,
                                                          (float2*)c.d_u + v * vs);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c.stream));
  return 0;
}

static int full_var_get(Ctx& c, int which, int v, double* host) {
  const size_t fs = full_elems(c), vs = (size_t)c.g.xz_tot * c.n;
  if (fs * sizeof(double2) > c.uz_elems * c.csz) return set_error("full-layout staging does not fit");
  const Geo g = make_geo(c);
  const void* src = which == PSDNS_FIELD_U ? c.d_u : c.d_un;
  CK(cudaMemsetAsync(c.d_uz, 0, sizeof(double2) * fs, c.stream));
  if (c.prec == PSDNS_PREC_FP64)
    k_cyl_to_full<double><<<148 * 8, 256, 0, c.stream>>>(g, (const double2*)src + v * vs, (double2*)c.d_uz);
  else
    k_cyl_to_full<float><<<148 * 8, 256, 0, c.stream>>>(g, (const float2*)src + v * vs, (double2*)c.d_uz);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, c.d_uz, sizeof(double2) * fs, cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return 0;
}

// big-endian Fortran record helpers for the checkpoint files
static void be32(std::vector<unsigned char>& b, uint32_t v) {
  for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
}
static void be64(unsigned char* p, double d) {
  uint64_t v;
  std::memcpy(&v, &d, 8);
  for (int i = 0; i < 8; i++) p[i] = (unsigned char)(v >> (56 - 8 * i));
}
static double rd_be64(const unsigned char* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
  double d;
  std::memcpy(&d, &v, 8);
  return d;
}
static uint32_t rd_be32(const unsigned char* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}
static bool write_record(FILE* f, const unsigned char* data, size_t bytes) {
  std::vector<unsigned char> m;
  be32(m, (uint32_t)bytes);
  return fwrite(m.data(), 1, 4, f) == 4 && fwrite(data, 1, bytes, f) == bytes && fwrite(m.data(), 1, 4, f) == 4;
}
static bool read_record(FILE* f, std::vector<unsigned char>& out) {
  unsigned char m[4];
  if (fread(m, 1, 4, f) != 4) return false;
  const uint32_t len = rd_be32(m);
  out.resize(len);
  if (fread(out.data(), 1, len, f) != len) return false;
  unsigned char m2[4];
  return fread(m2, 1, 4, f) == 4 && rd_be32(m2) == len;
}


}  // namespace psdns

using namespace psdns;

extern "C" {

int psdns_gpu_last_error(char* buf, int32_t len) {
  if (!buf || len <= 0) return 1;
  std::snprintf(buf, (size_t)len, "%s", g_last_error.c_str());
  return 0;
}

int psdns_gpu_default_params(psdns_params* p) {
  if (!p) return set_error("null params");
  std::memset(p, 0, sizeof *p);
  p->nx = p->ny = p->nz = 64;
  p->nc = 0;
  p->precision = PSDNS_PREC_FP32;
  p->kshift = 1;
  p->ksran = 1;
  p->seed_input = 122929298;   // PSDNS/input, iseed record
  p->kranf1 = 5;
  p->kranf2 = 5;
  p->viscos = 0.0028;
  p->beta1 = p->beta2 = p->beta3 = 1.0;
  p->cfl = 3.77;
  p->dt = 0.0;
  p->kforce = 0.0;
  p->tforce = 6.199433e-01;
  p->epsfor = 1.77063e-03;
  p->tfiuo = 0.4;
  p->pr = 1.0;
  return 0;
}

int psdns_gpu_geometry(int32_t n, int32_t* kxn, int32_t* xz_tot, int32_t* cut_z, int32_t* colstart) {
  if (n < 8 || (n & 1)) return set_error("grid size %d not supported", n);
  Geometry g;
  build_geometry(n, g);
  if (kxn) *kxn = g.kxn;
  if (xz_tot) *xz_tot = g.xz_tot;
  if (cut_z) for (int i = 0; i < g.kxn; i++) cut_z[i] = g.cut[i];
  if (colstart) for (int i = 0; i <= g.kxn; i++) colstart[i] = g.colstart[i];
  return 0;
}

int psdns_gpu_kymax(int32_t n, int32_t* kymax) {
  if (n < 8 || (n & 1)) return set_error("grid size %d not supported", n);
  if (!kymax) return set_error("null argument");
  Geometry g;
  build_geometry(n, g);
  for (int a = 0; a < g.xz_tot; a++) kymax[a] = g.kymax[a];
  return 0;
}

int psdns_gpu_init(const psdns_params* p, void** out) {
  if (!p || !out) return set_error("null argument");
  *out = nullptr;
  if (p->nx != p->ny || p->nx != p->nz) return set_error("only cubic boxes are supported (nx=ny=nz)");
  if (p->nc != 0 && p->nc != 1) return set_error("nc=%d: 0 or 1 passive scalars are supported", p->nc);
  if (p->nc == 1 && !(p->pr > 0.)) return set_error("Schmidt number pr must be positive");
  if (p->precision != PSDNS_PREC_FP32 && p->precision != PSDNS_PREC_FP64)
    return set_error("precision must be PSDNS_PREC_FP32 or PSDNS_PREC_FP64");
  if (p->kshift < 1 || p->kshift > 4) return set_error("kshift must be 1..4");
  if (p->ksran < 1 || p->ksran > 20 || p->kranf1 < 1 || p->kranf1 > 20 || p->kranf2 < 1 || p->kranf2 > 20)
    return set_error("RNG sequence numbers must be 1..20 (ranseq.f:131)");
  if (p->seed_input <= 0) return set_error("seed iseed=%d must be positive (ranu.f:33)", p->seed_input);
  if (p->cfl <= 0. && !(p->dt > 0.)) return set_error("fixed dt must be positive when cfl <= 0");
  if (p->rkmethod != 0 && p->rkmethod != 2 && p->rkmethod != 4)
    return set_error("rkmethod must be 2 or 4 (0: 2)");
  if (p->rkmethod == 4 && (p->nc != 0 || p->dft != PSDNS_DFT_FP32))
    return set_error("RK4 advances the velocity only (nc = 0) with the FP32 transforms");
  if (p->dft != PSDNS_DFT_FP32 && p->dft != PSDNS_DFT_TC_BF16X3)
    return set_error("dft must be PSDNS_DFT_FP32 or PSDNS_DFT_TC_BF16X3");
  if (p->dft == PSDNS_DFT_TC_BF16X3 && (p->precision != PSDNS_PREC_FP32 || p->nx != 1024))
    return set_error("the tensor-core transforms (PSDNS_DFT_TC_BF16X3) need an FP32 state at n = 1024");
  Ops o;
  if (!get_ops(p->precision, p->nx, p->nc, o))
    return set_error("grid size %d not supported (16..1024 powers of 2, 48, 96)", p->nx);
  Ctx* c = new Ctx();
  c->p = *p;
  c->n = p->nx;
  c->prec = p->precision;
  c->nc = p->nc;
  c->nv = 3 + p->nc;
  build_geometry(c->n, c->g);
  const int n = c->n;
  const bool dbl = c->prec == PSDNS_PREC_FP64;
  c->csz = dbl ? sizeof(double2) : sizeof(float2);
  const int tbi = dbl ? Tiles<double>::TB_I : Tiles<float>::TB_I;
  const int tbf = dbl ? Tiles<double>::TB_F : Tiles<float>::TB_F;
  const int tz = dbl ? Tiles<double>::TZ : Tiles<float>::TZ;
  c->nzt = n / tz;
  c->nab_i = (c->g.xz_tot + tbi - 1) / tbi;
  c->nab_f = (c->g.xz_tot + tbf - 1) / tbf;
  // ub: 3 + 2 nc backward variables (TB_I blocks) or 4 + nc forward terms
  // (TB_F blocks); uz: 5 + nc slots (3 + 3 nc inputs, 5 + nc outputs)
  const size_t ubi = dbl ? ubi_var_elems<double>(c->nab_i, n) : ubi_var_elems<float>(c->nab_i, n);
  c->ub_elems = std::max((size_t)(3 + 2 * c->nc) * ubi, (size_t)(4 + c->nc) * (dbl ? ubf_var_elems<double>(c->nab_f, n) : ubf_var_elems<float>(c->nab_f, n)));
  c->uz_elems = (size_t)(5 + c->nc) * n * n * c->g.kxn;
  c->st_elems = (size_t)c->nv * c->g.xz_tot * n;
  c->rng.init(p->seed_input);
  c->dt0 = p->dt;
  c->dt = p->dt;
  // forcing dimensions (param_set.f:33,37)
  c->kfor = (int)(p->kforce / std::min(p->beta1, p->beta2 + p->beta3) + 1.5);
  c->k2fo = 2 * c->kfor - 1;
  auto fail = [&](int rc) { psdns_gpu_finalize(c); return rc; };
  size_t need = c->csz * (2 * c->st_elems + c->ub_elems + c->uz_elems);
  size_t freeb = 0, totb = 0;
  if (cudaMemGetInfo(&freeb, &totb) != cudaSuccess) { delete c; return set_error("no CUDA device available"); }
  if (need + (size_t)256 * 1024 * 1024 > freeb) {
    delete c;
    return set_error("need %.2f GB of device memory, %.2f GB free", need / 1e9, freeb / 1e9);
  }
  if (o.setup()) return fail(1);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(set_error("stream"));
  const Geometry& g = c->g;
#define ALLOC(ptr, bytes) if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) return fail(set_error("cudaMalloc of %zu bytes failed", (size_t)(bytes)))
  ALLOC(c->d_colstart, sizeof(int) * (g.kxn + 1));
  ALLOC(c->d_ax, sizeof(int) * g.xz_tot);
  ALLOC(c->d_az, sizeof(int) * g.xz_tot);
  ALLOC(c->d_kymax, sizeof(int) * g.xz_tot);
  ALLOC(c->d_u, c->csz * c->st_elems);
  ALLOC(c->d_un, c->csz * c->st_elems);
  ALLOC(c->d_ub, c->csz * c->ub_elems);
  ALLOC(c->d_uz, c->csz * c->uz_elems);
  const size_t tabb = dbl ? TabLayout<double>(n).total : TabLayout<float>(n).total;
  ALLOC(c->d_tabs, tabb);
  ALLOC(c->d_velmax, sizeof(unsigned long long));
  const size_t nfor = (size_t)c->kfor * c->k2fo * c->k2fo * 3;
  ALLOC(c->d_forc, c->csz * std::max<size_t>(nfor, 1));
  ALLOC(c->d_efkz, sizeof(double) * 3 * (n / 2 + 2));
#undef ALLOC
#define ALLOC2(ptr, bytes) if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) return fail(set_error("cudaMalloc of %zu bytes failed", (size_t)(bytes)))
  if (cudaMallocHost(&c->h_tabs, tabb) != cudaSuccess) return fail(set_error("cudaMallocHost"));
  if (cudaMallocHost((void**)&c->h_velmax, sizeof(unsigned long long)) != cudaSuccess) return fail(set_error("cudaMallocHost"));
  if (cudaMallocHost(&c->h_forc, c->csz * std::max<size_t>(nfor, 1)) != cudaSuccess) return fail(set_error("cudaMallocHost"));
  c->forcing.setup(c->kfor, n, p->kforce, p->tforce, p->epsfor, p->tfiuo, p->kranf1, p->kranf2,
                   p->beta1 * p->beta1, p->beta2 * p->beta2, p->beta3 * p->beta3);
  std::memset(c->h_tabs, 0, tabb);
  if (cudaMemcpy(c->d_colstart, g.colstart.data(), sizeof(int) * (g.kxn + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_ax, g.ax.data(), sizeof(int) * g.xz_tot, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_az, g.az.data(), sizeof(int) * g.xz_tot, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_kymax, g.kymax.data(), sizeof(int) * g.xz_tot, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(set_error("geometry upload failed"));
  if (o.twiddles(*c)) return fail(1);
  c->dft = p->dft;
  c->rk = p->rkmethod == 4 ? 4 : 2;
  if (c->rk == 4) {
    ALLOC2(c->d_u1, c->csz * c->st_elems);
    if (cudaMemset(c->d_u1, 0, c->csz * c->st_elems) != cudaSuccess) return fail(set_error("memset failed"));
  }
  if (c->dft == PSDNS_DFT_TC_BF16X3) {
    std::vector<uint16_t> bt(tc::kBBytes / 2);
    std::vector<float2> tw2(1024);
    tc::build_tables(bt.data(), tw2.data());
    ALLOC2(c->d_tcb, tc::kBBytes);
    ALLOC2(c->d_tw2, sizeof(float2) * 1024);
    ALLOC2(c->d_tcerr, sizeof(unsigned));
    if (cudaMemcpy(c->d_tcb, bt.data(), tc::kBBytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_tw2, tw2.data(), sizeof(float2) * 1024, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(c->d_tcerr, 0, sizeof(unsigned)) != cudaSuccess)
      return fail(set_error("tensor-core table upload failed"));
  }
  {
    // cubic B-spline symbol per axis: 6 / (4 + 2 cos(2 pi k / n))
    const size_t ns = (size_t)(n / 2 + 1) + 2 * n;
    std::vector<double> f(ns);
    const double pi = 4. * std::atan(1.);
    for (int x = 0; x <= n / 2; x++) f[x] = 6. / (4. + 2. * std::cos(2. * pi * x / n));
    for (int y = 0; y < n; y++) f[n / 2 + 1 + y] = 6. / (4. + 2. * std::cos(2. * pi * g.ky[y] / n));
    for (int z = 0; z < n; z++) f[n / 2 + 1 + n + z] = 6. / (4. + 2. * std::cos(2. * pi * g.kz[z] / n));
    const size_t rsz = dbl ? sizeof(double) : sizeof(float);
    ALLOC2(c->d_spf, rsz * ns);
    std::vector<float> ff(ns);
    for (size_t i = 0; i < ns; i++) ff[i] = (float)f[i];
    if (cudaMemcpy(c->d_spf, dbl ? (const void*)f.data() : (const void*)ff.data(), rsz * ns,
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(set_error("prefilter upload failed"));
  }
  if (cudaMemset(c->d_u, 0, c->csz * c->st_elems) != cudaSuccess ||
      cudaMemset(c->d_un, 0, c->csz * c->st_elems) != cudaSuccess ||
      cudaMemset(c->d_forc, 0, c->csz * std::max<size_t>(nfor, 1)) != cudaSuccess ||
      cudaMemset(c->d_efkz, 0, sizeof(double) * 3 * (n / 2 + 2)) != cudaSuccess)
    return fail(set_error("memset failed"));
  *out = c;
  return 0;
}

int psdns_gpu_finalize(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return 0;
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->d_colstart, c->d_ax, c->d_az, c->d_kymax, c->d_tw, c->d_tabs, c->d_u, c->d_un,
                  c->d_ub, c->d_uz, c->d_forc, c->d_efkz, c->d_velmax, c->d_pos, c->d_vel, c->d_bs, c->d_spf,
                  c->d_tcb, c->d_tw2, c->d_tcerr, c->d_shf, c->d_u1};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (int s = 0; s < 4; s++)
    for (int k = 0; k < 6; k++)
      for (int e = 0; e < 2; e++)
        if (c->ev[s][k][e]) cudaEventDestroy(c->ev[s][k][e]);
  if (c->s_in) cudaStreamSynchronize(c->s_in);
  if (c->s_out) cudaStreamSynchronize(c->s_out);
  for (int k = 0; k < Ctx::kChunks; k++) {
    cudaEvent_t* evs[] = {&c->ev_h2d[k], &c->ev_conv_in[k], &c->ev_conv_out[k], &c->ev_d2h[k]};
    for (cudaEvent_t* e : evs)
      if (*e) cudaEventDestroy(*e);
  }
  if (c->ev_ready) cudaEventDestroy(c->ev_ready);
  if (c->d_in_stage) cudaFree(c->d_in_stage);
  if (c->d_out_stage) cudaFree(c->d_out_stage);
  if (c->s_in) cudaStreamDestroy(c->s_in);
  if (c->s_out) cudaStreamDestroy(c->s_out);
  if (c->h_tabs) cudaFreeHost(c->h_tabs);
  if (c->h_velmax) cudaFreeHost(c->h_velmax);
  if (c->h_forc) cudaFreeHost(c->h_forc);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int psdns_gpu_set_state_async(void* ctx, const double* un, int32_t layout) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !un) return set_error("null argument");
  if (layout != PSDNS_LAYOUT_YCYL) return set_error("asynchronous state copies use PSDNS_LAYOUT_YCYL");
  if (async_setup(*c)) return 1;
  const char* h = (const char*)un;
  const size_t bytes = sizeof(double2) * c->st_elems;
  // chunks of a pending sphere download do not match these chunks
  const bool same = c->pend_out == h && c->pend_out_bytes == bytes && !c->pend_sphere;
  const bool overlap = c->pend_out && h < c->pend_out + c->pend_out_bytes && c->pend_out < h + bytes;
  double2* stage = (double2*)c->d_in_stage;
  for (int k = 0; k < Ctx::kChunks; k++) {
    size_t off, cnt;
    chunk_range(*c, k, off, cnt);
    if (!cnt) continue;
    // the staging chunk is free once the previous upload's conversion read it
    if (c->in_pending) CK(cudaStreamWaitEvent(c->s_in, c->ev_conv_in[k], 0));
    if (same) {
      CK(cudaStreamWaitEvent(c->s_in, c->ev_d2h[k], 0));
    } else if (overlap) {
      for (int j = 0; j < Ctx::kChunks; j++) CK(cudaStreamWaitEvent(c->s_in, c->ev_d2h[j], 0));
    }
    CK(cudaMemcpyAsync(stage + off, h + off * sizeof(double2), cnt * sizeof(double2), cudaMemcpyHostToDevice,
                       c->s_in));
    CK(cudaEventRecord(c->ev_h2d[k], c->s_in));
    CK(cudaStreamWaitEvent(c->stream, c->ev_h2d[k], 0));
    if (c->prec == PSDNS_PREC_FP64)
      k_from_f64<double><<<148 * 4, 256, 0, c->stream>>>(stage + off, (double2*)c->d_un + off,
                                                          (double2*)c->d_u + off, cnt);
    else
      k_from_f64<float><<<148 * 4, 256, 0, c->stream>>>(stage + off, (float2*)c->d_un + off, (float2*)c->d_u + off,
                                                         cnt);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev_conv_in[k], c->stream));
  }
  c->in_pending = true;
  return 0;
}

int psdns_gpu_get_state_async(void* ctx, double* out, int32_t which, int32_t layout) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !out) return set_error("null argument");
  if (layout != PSDNS_LAYOUT_YCYL) return set_error("asynchronous state copies use PSDNS_LAYOUT_YCYL");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  if (async_setup(*c)) return 1;
  const void* src = which == PSDNS_FIELD_U ? c->d_u : c->d_un;
  double2* stage = (double2*)c->d_out_stage;
  const bool had = c->pend_out != nullptr;
  for (int k = 0; k < Ctx::kChunks; k++) {
    size_t off, cnt;
    chunk_range(*c, k, off, cnt);
    if (!cnt) continue;
    // the staging chunk is free once the previous download of it finished
    if (had) CK(cudaStreamWaitEvent(c->stream, c->ev_d2h[k], 0));
    if (c->prec == PSDNS_PREC_FP64)
      k_to_f64<double><<<148 * 4, 256, 0, c->stream>>>((const double2*)src + off, stage + off, cnt);
    else
      k_to_f64<float><<<148 * 4, 256, 0, c->stream>>>((const float2*)src + off, stage + off, cnt);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev_conv_out[k], c->stream));
    CK(cudaStreamWaitEvent(c->s_out, c->ev_conv_out[k], 0));
    CK(cudaMemcpyAsync((char*)out + off * sizeof(double2), stage + off, cnt * sizeof(double2),
                       cudaMemcpyDeviceToHost, c->s_out));
    CK(cudaEventRecord(c->ev_d2h[k], c->s_out));
  }
  c->pend_out = (const char*)out;
  c->pend_out_bytes = sizeof(double2) * c->st_elems;
  c->pend_sphere = false;
  return 0;
}

// device address of pinned (page-locked, mapped) host memory, or an error
static int mapped_host(const void* p, void** dptr) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return set_error("host array: pointer attributes unavailable");
  }
  if (at.type != cudaMemoryTypeHost || !at.devicePointer)
    return set_error("sphere copies need pinned host memory (cudaHostAlloc or cudaHostRegister)");
  *dptr = at.devicePointer;
  return 0;
}

// columns of chunk k of the sphere copies
static void sphere_chunk(const Ctx& c, int k, int& a0, int& a1) {
  const long long tot = c.g.xz_tot;
  a0 = (int)(tot * k / Ctx::kChunks);
  a1 = (int)(tot * (k + 1) / Ctx::kChunks);
}

int psdns_gpu_host_register(void* ptr, size_t bytes) {
  if (!ptr || bytes == 0) return set_error("null or empty host array");
  const cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error("cudaHostRegister: %s", cudaGetErrorString(e));
  }
  return 0;
}

int psdns_gpu_host_unregister(void* ptr) {
  if (!ptr) return set_error("null host array");
  const cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error("cudaHostUnregister: %s", cudaGetErrorString(e));
  }
  return 0;
}

int psdns_gpu_set_state_sphere_async(void* ctx, const double* un) {
  Ctx* c = (Ctx*)ctx;
  touch(c, true);
  if (!c || !un) return set_error("null argument");
  if (async_setup(*c, false)) return 1;
  void* dh = nullptr;
  if (mapped_host(un, &dh)) return 1;
  // directly after a sphere download: that download already waited for the
  // state (ev_ready), and chunk k waits for its chunk k only; otherwise wait
  // for everything enqueued so far
  const bool follow = c->sphere_get_pending && c->sphere_get_call == c->api_calls - 1;
  if (!follow) {
    if (c->sphere_get_pending)
      for (int k = 0; k < Ctx::kChunks; k++) CK(cudaStreamWaitEvent(c->s_in, c->ev_d2h[k], 0));
    CK(cudaEventRecord(c->ev_ready, c->stream));
  }
  if (c->pend_out && !c->sphere_get_pending)   // a pending full-array download
    for (int k = 0; k < Ctx::kChunks; k++) CK(cudaStreamWaitEvent(c->s_in, c->ev_d2h[k], 0));
  CK(cudaStreamWaitEvent(c->s_in, c->ev_ready, 0));
  const Geo g = make_geo(*c);
  for (int k = 0; k < Ctx::kChunks; k++) {
    int a0, a1;
    sphere_chunk(*c, k, a0, a1);
    if (follow) CK(cudaStreamWaitEvent(c->s_in, c->ev_d2h[k], 0));
    if (a1 > a0) {
      // two blocks per SM (reads wait on the bus), leaving room for the
      // download of another chunk beside it
      const int blocks = std::min(2 * 148, (a1 - a0 + 7) / 8);
      if (c->prec == PSDNS_PREC_FP64)
        k_sphere_in<double><<<blocks, 256, 0, c->s_in>>>(g, c->nv, (const double2*)dh, (double2*)c->d_un,
                                                         (double2*)c->d_u, a0, a1);
      else
        k_sphere_in<float><<<blocks, 256, 0, c->s_in>>>(g, c->nv, (const double2*)dh, (float2*)c->d_un,
                                                        (float2*)c->d_u, a0, a1);
      CK(cudaGetLastError());
    }
    CK(cudaEventRecord(c->ev_h2d[k], c->s_in));
    CK(cudaStreamWaitEvent(c->stream, c->ev_h2d[k], 0));
  }
  // the context stream now follows every chunk, and so every download chunk
  c->sphere_get_pending = false;
  c->pend_out = nullptr;
  c->pend_out_bytes = 0;
  return 0;
}

int psdns_gpu_get_state_sphere_async(void* ctx, double* out, int32_t which) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !out) return set_error("null argument");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  if (async_setup(*c, false)) return 1;
  void* dh = nullptr;
  if (mapped_host(out, &dh)) return 1;
  // a pending full-array download of the staging buffers must not be
  // overtaken; the state is ready when the context stream reaches ev_ready
  if (c->pend_out)
    for (int k = 0; k < Ctx::kChunks; k++) CK(cudaStreamWaitEvent(c->s_out, c->ev_d2h[k], 0));
  CK(cudaEventRecord(c->ev_ready, c->stream));
  CK(cudaStreamWaitEvent(c->s_out, c->ev_ready, 0));
  const Geo g = make_geo(*c);
  const void* src = which == PSDNS_FIELD_U ? c->d_u : c->d_un;
  for (int k = 0; k < Ctx::kChunks; k++) {
    int a0, a1;
    sphere_chunk(*c, k, a0, a1);
    if (a1 > a0) {
      const int blocks = std::min(148, (a1 - a0 + 7) / 8);
      if (c->prec == PSDNS_PREC_FP64)
        k_sphere_out<double><<<blocks, 256, 0, c->s_out>>>(g, c->nv, (const double2*)src, (double2*)dh, a0, a1);
      else
        k_sphere_out<float><<<blocks, 256, 0, c->s_out>>>(g, c->nv, (const float2*)src, (double2*)dh, a0, a1);
      CK(cudaGetLastError());
    }
    CK(cudaEventRecord(c->ev_d2h[k], c->s_out));
  }
  c->sphere_get_pending = true;
  c->sphere_get_call = c->api_calls;
  c->pend_out = (const char*)out;
  c->pend_out_bytes = sizeof(double2) * c->st_elems;
  c->pend_sphere = true;
  return 0;
}

int psdns_gpu_sync(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (c->s_in) {
    CK(cudaStreamSynchronize(c->s_in));
    CK(cudaStreamSynchronize(c->s_out));
  }
  CK(cudaStreamSynchronize(c->stream));
  c->pend_out = nullptr;
  c->pend_out_bytes = 0;
  c->in_pending = false;
  return 0;
}

// host (complex double, YCYL) -> device state, through ub as staging
// ---------------------------------------------------------------------------
// Checkpoint files in the reference's single-task pencil format
// (homogeneous/outpen_write_r.f, compiled with -fconvert=big-endian and
// -fdefault-real-8, makefile:249-256): Fortran unformatted sequential
// records with 4-byte big-endian length markers; per variable i = 1..3+nc
// the records (i, nx, ny, nz), (xist, xisz, zjst, zjsz, 1, ny) as int32,
// then for every z but the Nyquist plane two records of real(8) pairs
// (re, im) with x fastest: rows y = 1..ny/2, then y = ny/2+2..ny.  One task
// holds kx = 0..nx/2-1 (xisz = nx/2, mpisetup.f:179) and every z.
// ---------------------------------------------------------------------------
int psdns_gpu_write_checkpoint(void* ctx, const char* path, int32_t which) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !path) return set_error("null argument");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  const int n = c->n, nxh = n / 2 + 1, xisz = n / 2;
  const size_t fs = (size_t)nxh * n * n;
  // one variable of the full spectrum on the host at a time
  std::vector<double> full;
  std::vector<unsigned char> rec, row;
  try {
    full.resize(2 * fs);
    row.resize((size_t)16 * xisz * (n / 2));
  } catch (const std::bad_alloc&) {
    return set_error("checkpoint: cannot allocate %.2f GB of host memory", 16.0 * fs / 1e9);
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error("cannot open %s for writing", path);
  bool ok = true;
  for (int v = 0; v < c->nv && ok; v++) {
    if (full_var_get(*c, which, v, full.data())) { std::fclose(f); return 1; }
    rec.clear();
    for (uint32_t x : {(uint32_t)(v + 1), (uint32_t)n, (uint32_t)n, (uint32_t)n}) be32(rec, x);
    ok = ok && write_record(f, rec.data(), rec.size());
    rec.clear();
    for (uint32_t x : {1u, (uint32_t)xisz, 1u, (uint32_t)n, 1u, (uint32_t)n}) be32(rec, x);
    ok = ok && write_record(f, rec.data(), rec.size());
    const double* u = full.data();
    for (int z = 0; z < n && ok; z++) {
      if (z == n / 2) continue;   // nzhp
      for (int half = 0; half < 2 && ok; half++) {
        const int y0 = half == 0 ? 0 : n / 2 + 1, y1 = half == 0 ? n / 2 : n;
        size_t o = 0;
        for (int y = y0; y < y1; y++)
          for (int x = 0; x < xisz; x++) {
            const double* e = u + 2 * (((size_t)z * n + y) * nxh + x);
            be64(&row[o], e[0]);
            be64(&row[o + 8], e[1]);
            o += 16;
          }
        ok = write_record(f, row.data(), o);
      }
    }
  }
  if (std::fclose(f) != 0) ok = false;
  return ok ? 0 : set_error("write to %s failed", path);
}

int psdns_gpu_read_checkpoint(void* ctx, const char* path) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !path) return set_error("null argument");
  const int n = c->n, nxh = n / 2 + 1, xisz = n / 2;
  const size_t fs = (size_t)nxh * n * n;
  std::vector<double> full;
  try {
    full.resize(2 * fs);
  } catch (const std::bad_alloc&) {
    return set_error("checkpoint: cannot allocate %.2f GB of host memory", 16.0 * fs / 1e9);
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error("cannot open %s", path);
  std::vector<unsigned char> rec;
  int err = 0;
  for (int v = 0; v < c->nv && !err; v++) {
    std::fill(full.begin(), full.end(), 0.0);
    if (!read_record(f, rec) || rec.size() != 16) { err = set_error("%s: bad header of variable %d", path, v + 1); break; }
    if ((int)rd_be32(&rec[0]) != v + 1 || (int)rd_be32(&rec[4]) != n || (int)rd_be32(&rec[8]) != n ||
        (int)rd_be32(&rec[12]) != n) {
      err = set_error("%s: variable %d is not a %d^3 field", path, v + 1, n);
      break;
    }
    if (!read_record(f, rec) || rec.size() != 24 || rd_be32(&rec[0]) != 1 || (int)rd_be32(&rec[4]) != xisz ||
        rd_be32(&rec[8]) != 1 || (int)rd_be32(&rec[12]) != n) {
      err = set_error("%s: not a single-task pencil (xist 1, xisz %d, zjst 1, zjsz %d)", path, xisz, n);
      break;
    }
    double* u = full.data();
    for (int z = 0; z < n && !err; z++) {
      if (z == n / 2) continue;
      for (int half = 0; half < 2; half++) {
        const int y0 = half == 0 ? 0 : n / 2 + 1, y1 = half == 0 ? n / 2 : n;
        if (!read_record(f, rec) || rec.size() != (size_t)16 * xisz * (y1 - y0)) {
          err = set_error("%s: short record at z = %d", path, z + 1);
          break;
        }
        size_t o = 0;
        for (int y = y0; y < y1; y++)
          for (int x = 0; x < xisz; x++) {
            double* e = u + 2 * (((size_t)z * n + y) * nxh + x);
            e[0] = rd_be64(&rec[o]);
            e[1] = rd_be64(&rec[o + 8]);
            o += 16;
          }
      }
    }
    if (!err && full_var_set(*c, v, full.data())) err = 1;
  }
  std::fclose(f);
  return err;
}

// ---------------------------------------------------------------------------
// Checkpoint metadata (store.f, ranseq.f) and multi-task pencil sets
// (homogeneous/outpen_write_r.f, inpen_read_r.f)
// ---------------------------------------------------------------------------
// store.f:347-348: format 900 = (10i8), format 910 = (1p,5e15.8)
static bool fmt_ints(FILE* f, const std::vector<long long>& v, int per, int w) {
  for (size_t i = 0; i < v.size(); i++) {
    if (std::fprintf(f, "%*lld", w, v[i]) < 0) return false;
    if ((i + 1) % per == 0 || i + 1 == v.size())
      if (std::fputc('\n', f) == EOF) return false;
  }
  return true;
}
static bool fmt_reals(FILE* f, const std::vector<double>& v) {
  for (size_t i = 0; i < v.size(); i++) {
    if (std::fprintf(f, "%15.8E", v[i]) < 0) return false;
    if ((i + 1) % 5 == 0 || i + 1 == v.size())
      if (std::fputc('\n', f) == EOF) return false;
  }
  return true;
}
// fixed-width fields, `per` to a line (Fortran list of a repeated format)
static bool read_fields(FILE* f, size_t count, int per, int w, std::vector<std::string>& out) {
  out.clear();
  char line[4096];
  while (out.size() < count) {
    if (!std::fgets(line, sizeof line, f)) return false;
    std::string l(line);
    while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
    for (int k = 0; k < per && out.size() < count; k++) {
      if ((size_t)(k + 1) * w > l.size()) {
        if ((size_t)k * w >= l.size()) break;
      }
      out.push_back(l.substr((size_t)k * w, (size_t)w));
    }
  }
  return true;
}
static bool parse_real(const std::string& s, double& d) {
  std::string t = s;
  for (char& ch : t)
    if (ch == 'D' || ch == 'd') ch = 'E';
  char* e = nullptr;
  d = std::strtod(t.c_str(), &e);
  return e != t.c_str();
}

// the store.f record of a context: isdata (icall 1 then istep), rsdata
// (icall 1 then time, gsh(:,2), b11 b22 b33 b12 (2 each), suo, svo)
static void store_data(const Ctx& c, int istep, int iostep, std::vector<long long>& is, int& nic2,
                       std::vector<double>& rs, int& nrc2) {
  const psdns_params& p = c.p;
  const int ncd = p.nc == 0 ? 1 : p.nc;   // param_set.f:19-24
  // my, mz, nxhvs, nyvs, nzvs are locals that store.f never sets; 0 here
  is = {p.nx, p.ny, p.nz, 0, 0, 0, 0, 0, p.nc, ncd, c.kfor, iostep, p.kshift};
  nic2 = (int)is.size();
  is.push_back(istep);
  rs.clear();
  rs.push_back(p.viscos);
  for (int i = 0; i < ncd; i++) rs.push_back(p.pr);
  for (int i = 0; i < 4; i++) rs.push_back(0.0);   // a11, a22, a33, shear
  for (int i = 0; i < ncd; i++)
    for (int j = 0; j < 3; j++) rs.push_back(p.grad[j]);
  for (double v : {p.beta1, p.beta2, p.beta3, p.cfl, c.dt, p.tforce, p.epsfor, p.kforce, p.tfiuo}) rs.push_back(v);
  nrc2 = (int)rs.size();
  rs.push_back(c.time);
  for (int i = 0; i < 3; i++) rs.push_back(c.gsh[i][1]);
  for (double b : {p.beta1 * p.beta1, p.beta2 * p.beta2, p.beta3 * p.beta3, 0.0}) {
    rs.push_back(b);
    rs.push_back(b);
  }
  const int nrproc = c.forcing.nrproc;
  for (int i = 0; i < nrproc; i++) rs.push_back(c.forcing.suo[i]);
  for (int i = 0; i < nrproc; i++) rs.push_back(c.forcing.svo[i]);
}

int psdns_gpu_write_chkptou(void* ctx, const char* path, int32_t istep, int32_t iostep) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !path) return set_error("null argument");
  std::vector<long long> is;
  std::vector<double> rs;
  int nic2 = 0, nrc2 = 0;
  store_data(*c, istep, iostep, is, nic2, rs, nrc2);
  FILE* f = std::fopen(path, "w");
  if (!f) return set_error("cannot open %s for writing", path);
  bool ok = fmt_ints(f, {nic2, nrc2, (long long)is.size(), (long long)rs.size()}, 10, 8) && fmt_ints(f, is, 10, 8) &&
            fmt_reals(f, rs);
  if (std::fclose(f) != 0) ok = false;
  return ok ? 0 : set_error("write to %s failed", path);
}

int psdns_gpu_read_chkptou(void* ctx, const char* path, int32_t strict, int32_t* istep) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !path) return set_error("null argument");
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error("cannot open %s", path);
  std::vector<std::string> fld;
  long long hdr[4] = {0, 0, 0, 0};
  bool ok = read_fields(f, 4, 10, 8, fld);
  for (int i = 0; ok && i < 4; i++) hdr[i] = std::atoll(fld[i].c_str());
  std::vector<long long> ird;
  std::vector<double> rrd;
  if (ok) ok = hdr[2] > 0 && hdr[2] < 100 && hdr[3] > 0 && hdr[3] < 100000000 && read_fields(f, hdr[2], 10, 8, fld);
  if (ok) for (auto& x : fld) ird.push_back(std::atoll(x.c_str()));
  if (ok) ok = read_fields(f, hdr[3], 5, 15, fld);
  if (ok)
    for (auto& x : fld) {
      double d;
      if (!parse_real(x, d)) { ok = false; break; }
      rrd.push_back(d);
    }
  std::fclose(f);
  if (!ok) return set_error("%s: not a chkptou file (store.f formats 900/910)", path);
  std::vector<long long> is;
  std::vector<double> rs;
  int nic2 = 0, nrc2 = 0;
  store_data(*c, 0, 0, is, nic2, rs, nrc2);
  if (hdr[0] != nic2 || hdr[1] != nrc2 || (long long)ird.size() != (long long)is.size() ||
      (long long)rrd.size() != (long long)rs.size())
    return set_error("%s: %lld/%lld integers and %lld/%lld reals, this run stores %d/%zu and %d/%zu", path, hdr[0],
                     hdr[2], hdr[1], hdr[3], nic2, is.size(), nrc2, rs.size());
  if (strict) {
    // store.f:272-301 (kstop = 1): the stored parameters must be this run's;
    // the unset locals (3..7) and iostep (11) are not compared, reals to
    // the 9 digits of format 910
    for (int j = 0; j < nic2; j++) {
      if ((j >= 3 && j <= 7) || j == 11) continue;
      if (ird[j] != is[j]) return set_error("%s: integer no. %d is %lld, this run has %lld", path, j + 1, ird[j], is[j]);
    }
    for (int j = 0; j < nrc2; j++) {
      if (j == 1 + (c->p.nc == 0 ? 1 : c->p.nc) + 4 + 3 * (c->p.nc == 0 ? 1 : c->p.nc) + 4) continue;   // dt (cfl > 0: the last step's)
      if (std::fabs(rrd[j] - rs[j]) > 5e-9 * std::max(1.0, std::fabs(rs[j])))
        return set_error("%s: real no. %d is %.9g, this run has %.9g", path, j + 1, rrd[j], rs[j]);
    }
  }
  // store.f:303-320: istep0, time0, gsh(:,2), suo, svo
  size_t o = nrc2;
  c->time = rrd[o++];
  for (int i = 0; i < 3; i++) c->gsh[i][1] = rrd[o++];
  o += 8;
  const int nrproc = c->forcing.nrproc;
  for (int i = 0; i < nrproc; i++) c->forcing.suo[i] = rrd[o++];
  for (int i = 0; i < nrproc; i++) c->forcing.svo[i] = rrd[o++];
  c->jstep = 0;
  c->istart = 1;
  if (istep) *istep = (int32_t)ird[nic2];
  return 0;
}

int psdns_gpu_write_ranout(void* ctx, const char* path) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !path) return set_error("null argument");
  // ranseq.f:174-183 (k = -2): the active sequence's seed goes back into
  // its slot, then the 20 seeds are written with format (5i15)
  if (c->rng.ifst) c->rng.iseq[c->rng.klast - 1] = c->rng.iseed;
  else
    for (int i = 0; i < 20; i++) c->rng.iseq[i] = c->rng.seed_input;
  std::vector<long long> v(c->rng.iseq, c->rng.iseq + 20);
  FILE* f = std::fopen(path, "w");
  if (!f) return set_error("cannot open %s for writing", path);
  bool ok = fmt_ints(f, v, 5, 15);
  if (std::fclose(f) != 0) ok = false;
  return ok ? 0 : set_error("write to %s failed", path);
}

int psdns_gpu_read_ranin(void* ctx, const char* path) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !path) return set_error("null argument");
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error("cannot open %s", path);
  std::vector<std::string> fld;
  const bool ok = read_fields(f, 20, 5, 15, fld);
  std::fclose(f);
  if (!ok) return set_error("%s: not a ranout file (20 seeds, format 5i15)", path);
  // ranseq.f:83-118 (first call with k = -1): the table is read, the
  // active sequence is the first
  for (int i = 0; i < 20; i++) c->rng.iseq[i] = (int32_t)std::atoll(fld[i].c_str());
  c->rng.ifst = 1;
  c->rng.klast = 1;
  c->rng.iseed = c->rng.iseq[0];
  return 0;
}

// one variable's records of one pencil (outpen_write_r.f:62-72)
static bool pencil_write(FILE* f, int v, int n, const double* u, int xist, int xisz, int zjst, int zjsz,
                         std::vector<unsigned char>& row) {
  const int nxh = n / 2 + 1;
  std::vector<unsigned char> rec;
  for (uint32_t x : {(uint32_t)(v + 1), (uint32_t)n, (uint32_t)n, (uint32_t)n}) be32(rec, x);
  bool ok = write_record(f, rec.data(), rec.size());
  rec.clear();
  for (uint32_t x : {(uint32_t)xist, (uint32_t)xisz, (uint32_t)zjst, (uint32_t)zjsz, 1u, (uint32_t)n}) be32(rec, x);
  ok = ok && write_record(f, rec.data(), rec.size());
  for (int zp = 0; zp < zjsz && ok; zp++) {
    const int z = zjst - 1 + zp;
    if (z == n / 2) continue;   // nzhp
    for (int half = 0; half < 2 && ok; half++) {
      const int y0 = half == 0 ? 0 : n / 2 + 1, y1 = half == 0 ? n / 2 : n;
      size_t o = 0;
      for (int y = y0; y < y1; y++)
        for (int x = xist - 1; x < xist - 1 + xisz; x++) {
          const double* e = u + 2 * (((size_t)z * n + y) * nxh + x);
          be64(&row[o], e[0]);
          be64(&row[o + 8], e[1]);
          o += 16;
        }
      ok = write_record(f, row.data(), o);
    }
  }
  return ok;
}

int psdns_gpu_write_checkpoint_set(void* ctx, const char* prefix, int32_t iproc, int32_t jproc, int32_t which) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !prefix) return set_error("null argument");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  const int n = c->n, xh = n / 2;
  if (iproc < 1 || jproc < 1 || xh % iproc || n % jproc || iproc * jproc > 4096)
    return set_error("checkpoint set: iproc must divide n/2 = %d and jproc n = %d (at most 4096 tasks)", xh, n);
  const int xisz = xh / iproc, zjsz = n / jproc, nt = iproc * jproc;
  std::vector<double> full;
  std::vector<unsigned char> row;
  try {
    full.resize(2 * full_elems(*c));
    row.resize((size_t)16 * xisz * (n / 2));
  } catch (const std::bad_alloc&) {
    return set_error("checkpoint: cannot allocate %.2f GB of host memory", 16.0 * full_elems(*c) / 1e9);
  }
  // task t = jp * iproc + ip holds x in [ip xisz, (ip+1) xisz), z in [jp zjsz, (jp+1) zjsz)
  std::vector<FILE*> fs(nt, nullptr);
  int err = 0;
  for (int t = 0; t < nt && !err; t++) {
    const std::string fn = std::string(prefix) + ".p" + std::to_string(t);
    fs[t] = std::fopen(fn.c_str(), "wb");
    if (!fs[t]) err = set_error("cannot open %s for writing", fn.c_str());
  }
  for (int v = 0; v < c->nv && !err; v++) {
    if (full_var_get(*c, which, v, full.data())) { err = 1; break; }
    for (int t = 0; t < nt && !err; t++) {
      const int ip = t % iproc, jp = t / iproc;
      if (!pencil_write(fs[t], v, n, full.data(), ip * xisz + 1, xisz, jp * zjsz + 1, zjsz, row))
        err = set_error("write of %s.p%d failed", prefix, t);
    }
  }
  for (FILE* f : fs)
    if (f && std::fclose(f) != 0 && !err) err = set_error("closing a pencil file of %s failed", prefix);
  return err;
}

int psdns_gpu_read_checkpoint_set(void* ctx, const char* const* paths, int32_t nfiles) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !paths || nfiles < 1 || nfiles > 4096) return set_error("read_checkpoint_set: bad argument");
  const int n = c->n, nxh = n / 2 + 1, xh = n / 2;
  std::vector<double> full;
  std::vector<unsigned char> cover;
  try {
    full.resize(2 * full_elems(*c));
    cover.resize((size_t)xh * n);
  } catch (const std::bad_alloc&) {
    return set_error("checkpoint: cannot allocate %.2f GB of host memory", 16.0 * full_elems(*c) / 1e9);
  }
  std::vector<FILE*> fs(nfiles, nullptr);
  int err = 0;
  for (int t = 0; t < nfiles && !err; t++) {
    fs[t] = paths[t] ? std::fopen(paths[t], "rb") : nullptr;
    if (!fs[t]) err = set_error("cannot open pencil file %d (%s)", t, paths[t] ? paths[t] : "null");
  }
  std::vector<unsigned char> rec;
  for (int v = 0; v < c->nv && !err; v++) {
    std::fill(full.begin(), full.end(), 0.0);
    std::fill(cover.begin(), cover.end(), 0);
    for (int t = 0; t < nfiles && !err; t++) {
      FILE* f = fs[t];
      if (!read_record(f, rec) || rec.size() != 16 || (int)rd_be32(&rec[0]) != v + 1 ||
          (int)rd_be32(&rec[4]) != n || (int)rd_be32(&rec[8]) != n || (int)rd_be32(&rec[12]) != n) {
        err = set_error("%s: variable %d of a %d^3 field expected", paths[t], v + 1, n);
        break;
      }
      if (!read_record(f, rec) || rec.size() != 24) { err = set_error("%s: bad pencil header", paths[t]); break; }
      const int xist = (int)rd_be32(&rec[0]), xisz = (int)rd_be32(&rec[4]), zjst = (int)rd_be32(&rec[8]),
                zjsz = (int)rd_be32(&rec[12]);
      if (xist < 1 || xisz < 1 || xist - 1 + xisz > xh || zjst < 1 || zjsz < 1 || zjst - 1 + zjsz > n ||
          rd_be32(&rec[16]) != 1 || (int)rd_be32(&rec[20]) != n) {
        err = set_error("%s: pencil x %d+%d, z %d+%d outside the %d^3 box", paths[t], xist, xisz, zjst, zjsz, n);
        break;
      }
      for (int zp = 0; zp < zjsz && !err; zp++) {
        const int z = zjst - 1 + zp;
        if (z == n / 2) continue;
        for (int x = xist - 1; x < xist - 1 + xisz; x++) {
          if (cover[(size_t)x * n + z]++) { err = set_error("%s: x %d, z %d given twice", paths[t], x + 1, z + 1); break; }
        }
        for (int half = 0; half < 2 && !err; half++) {
          const int y0 = half == 0 ? 0 : n / 2 + 1, y1 = half == 0 ? n / 2 : n;
          if (!read_record(f, rec) || rec.size() != (size_t)16 * xisz * (y1 - y0)) {
            err = set_error("%s: short record at z = %d", paths[t], z + 1);
            break;
          }
          size_t o = 0;
          for (int y = y0; y < y1; y++)
            for (int x = xist - 1; x < xist - 1 + xisz; x++) {
              double* e = full.data() + 2 * (((size_t)z * n + y) * nxh + x);
              e[0] = rd_be64(&rec[o]);
              e[1] = rd_be64(&rec[o + 8]);
              o += 16;
            }
        }
      }
    }
    for (int x = 0; x < xh && !err; x++)
      for (int z = 0; z < n; z++)
        if (z != n / 2 && !cover[(size_t)x * n + z]) {
          err = set_error("the pencil set does not cover x %d, z %d", x + 1, z + 1);
          break;
        }
    if (!err && full_var_set(*c, v, full.data())) err = 1;
  }
  for (FILE* f : fs)
    if (f) std::fclose(f);
  return err;
}

int psdns_gpu_set_state(void* ctx, const double* un, int32_t layout) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !un) return set_error("null argument");
  if (layout != PSDNS_LAYOUT_YCYL && layout != PSDNS_LAYOUT_FULL) return set_error("unsupported layout %d", layout);
  const size_t vs = (size_t)c->g.xz_tot * c->n;
  if (layout == PSDNS_LAYOUT_FULL) {
    // one variable of the full half-complex array at a time, staged in uz
    const size_t fs = full_elems(*c);
    for (int v = 0; v < c->nv; v++)
      if (full_var_set(*c, v, un + 2 * v * fs)) return 1;
    return 0;
  }
  // stage one variable at a time: ub holds >= 2 variables of complex double
  for (int v = 0; v < c->nv; v++) {
    CK(cudaMemcpyAsync(c->d_ub, un + 2 * v * vs, sizeof(double2) * vs, cudaMemcpyHostToDevice, c->stream));
    const int blocks = 148 * 8;
    if (c->prec == PSDNS_PREC_FP64)
      k_from_f64<double><<<blocks, 256, 0, c->stream>>>((const double2*)c->d_ub, (double2*)c->d_un + v * vs,
                                                         (double2*)c->d_u + v * vs, vs);
    else
      k_from_f64<float><<<blocks, 256, 0, c->stream>>>((const double2*)c->d_ub, (float2*)c->d_un + v * vs,
                                                        (float2*)c->d_u + v * vs, vs);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int psdns_gpu_get_state(void* ctx, double* out, int32_t which, int32_t layout) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !out) return set_error("null argument");
  if (layout != PSDNS_LAYOUT_YCYL && layout != PSDNS_LAYOUT_FULL) return set_error("unsupported layout %d", layout);
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  const size_t vs = (size_t)c->g.xz_tot * c->n;
  void* src = which == PSDNS_FIELD_U ? c->d_u : c->d_un;
  if (layout == PSDNS_LAYOUT_FULL) {
    const size_t fs = full_elems(*c);
    for (int v = 0; v < c->nv; v++)
      if (full_var_get(*c, which, v, out + 2 * v * fs)) return 1;
    return 0;
  }
  for (int v = 0; v < c->nv; v++) {
    const int blocks = 148 * 8;
    if (c->prec == PSDNS_PREC_FP64)
      k_to_f64<double><<<blocks, 256, 0, c->stream>>>((const double2*)src + v * vs, (double2*)c->d_ub, vs);
    else
      k_to_f64<float><<<blocks, 256, 0, c->stream>>>((const float2*)src + v * vs, (double2*)c->d_ub, vs);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out + 2 * v * vs, c->d_ub, sizeof(double2) * vs, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int psdns_gpu_step(void* ctx, double* info) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  Ops o;
  if (!get_ops(c->prec, c->n, c->nc, o)) return set_error("bad context");
  c->jstep += 1;
  draw_shifts(*c);
  if (c->prec == PSDNS_PREC_FP64) fill_shift_tables<double>(*c); else fill_shift_tables<float>(*c);
  if (c->jstep == 1) {
    // factor tables are filled at stage 1; zero them before the first use
  }
  if (upload_tables(*c)) return 1;
  int ctl = 0;
  for (int k = 1; k <= c->rk; k++)
    if (run_stage(*c, o, k, &ctl)) return 1;
  CK(cudaStreamSynchronize(c->stream));
  prof_collect(*c, 0, 4, 5);
  for (int k = 1; k < c->rk; k++) prof_collect(*c, k, 0, 5);
  if (collect_forcing_stats(*c)) return 1;
  if (info) {
    info[0] = c->dt;
    info[1] = c->time;
    info[2] = c->velmax;
    info[3] = c->velmax * c->dt / 2. / (4. * std::atan(1.));
    info[4] = c->gsh[0][0];
    info[5] = c->gsh[1][0];
    info[6] = c->gsh[2][0];
    info[7] = (double)c->jstep;
  }
  return ctl ? 2 : 0;
}

int psdns_gpu_rk_stage(void* ctx, int32_t kstep, const double* gsh, const double* dt, const double* forcing,
                       double* velmax_out) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !gsh) return set_error("null argument");
  if (kstep < 1 || kstep > c->rk) return set_error("kstep must be 1 .. %d (rkmethod)", c->rk);
  if (forcing != nullptr && !(c->p.kforce > 0))
    return set_error("a forcing table was passed but the context was created with kforce = 0");
  Ops o;
  if (!get_ops(c->prec, c->n, c->nc, o)) return set_error("bad context");
  for (int i = 0; i < 3; i++) { c->gsh[i][0] = gsh[i]; c->gsh[i][1] = gsh[3 + i]; }
  if (c->prec == PSDNS_PREC_FP64) fill_shift_tables<double>(*c); else fill_shift_tables<float>(*c);
  if (kstep == 1) {
    if (!dt || !(*dt > 0)) return set_error("stage 1 needs a positive dt");
    c->dt = *dt;
    c->dt2 = c->dt / 2.;
    if (c->prec == PSDNS_PREC_FP64) fill_factor_tables<double>(*c); else fill_factor_tables<float>(*c);
    CK(cudaMemsetAsync(c->d_velmax, 0, sizeof(unsigned long long), c->stream));
    if (c->p.kforce > 0) CK(cudaMemsetAsync(c->d_efkz, 0, sizeof(double) * 3 * (c->n / 2 + 2), c->stream));
  }
  if (upload_tables(*c)) return 1;
  if (c->p.kforce > 0) {
    // the driver passes this step's table (force.f); none means zero forcing
    std::vector<double> zero;
    const double* tab = forcing;
    if (!tab) {
      zero.assign((size_t)2 * c->kfor * c->k2fo * c->k2fo * 3, 0.0);
      tab = zero.data();
    }
    if (kstep == 1 || forcing) { if (upload_forcing(*c, tab)) return 1; }
  }
  if (o.stage_a(*c, kstep)) return 1;
  if (kstep == 1) {
    CK(cudaMemcpyAsync(c->h_velmax, c->d_velmax, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(&c->velmax, c->h_velmax, sizeof(double));
    if (velmax_out) *velmax_out = c->velmax;
  }
  if (o.stage_b(*c, kstep)) return 1;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int psdns_gpu_field_init(void* ctx, int32_t seed) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (seed <= 0) return set_error("seed %d must be positive (ranu.f:33)", seed);
  const Geometry& g = c->g;
  const int n = c->n;
  if (c->nc > 0) {
    // the scalar starts from zero fluctuations (incond.f:49, kinit = 0)
    const size_t vs = (size_t)g.xz_tot * n;
    CK(cudaMemsetAsync((char*)c->d_u + 3 * vs * c->csz, 0, vs * c->csz, c->stream));
    CK(cudaMemsetAsync((char*)c->d_un + 3 * vs * c->csz, 0, vs * c->csz, c->stream));
  }
  // offsets of each column's first draw (in modes) in the traversal order
  std::vector<long long> off(g.xz_tot);
  long long acc = 0;
  for (int a = 0; a < g.xz_tot; a++) {
    off[a] = acc;
    const int km = std::min(g.kymax[a], n / 2 - 1);
    long long cnt = km >= 0 ? 2LL * km + 1 : 0;
    if (a == 0 && cnt > 0) cnt -= 1;   // the k = 0 mode draws nothing
    acc += cnt;
  }
  long long* d_off = nullptr;
  CK(cudaMalloc(&d_off, sizeof(long long) * g.xz_tot));
  cudaError_t e = cudaMemcpy(d_off, off.data(), sizeof(long long) * g.xz_tot, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(d_off); return set_error("upload failed: %s", cudaGetErrorString(e)); }
  Geo geo = make_geo(*c);
  const double s1 = c->p.beta1, s2 = c->p.beta2, s3 = c->p.beta3;

  const int kc0 = n / 2 - 1 - g.cut[0];
  if (c->prec == PSDNS_PREC_FP64) {
    k_field_init<double><<<148 * 8, 256, 0, c->stream>>>(geo, d_off, (uint32_t)seed, s1, s2, s3, (double2*)c->d_un,
                                                         (double2*)c->d_u);
    k_field_consym<double><<<148, 256, 0, c->stream>>>(n, kc0, g.xz_tot, (double2*)c->d_un, (double2*)c->d_u);
  } else {
    k_field_init<float><<<148 * 8, 256, 0, c->stream>>>(geo, d_off, (uint32_t)seed, s1, s2, s3, (float2*)c->d_un,
                                                        (float2*)c->d_u);
    k_field_consym<float><<<148, 256, 0, c->stream>>>(n, kc0, g.xz_tot, (float2*)c->d_un, (float2*)c->d_u);
  }
  e = cudaGetLastError();
  cudaError_t e2 = cudaStreamSynchronize(c->stream);
  cudaFree(d_off);
  if (e != cudaSuccess || e2 != cudaSuccess)
    return set_error("field init failed: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
  return 0;
}

int psdns_gpu_field_sinusoidal(void* ctx, double au, double av) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  const Geometry& g = c->g;
  const int n = c->n;
  if (g.kxn < 2) return set_error("grid too small for the sinusoidal field");
  // u = au sin x cos y cos z, v = av cos x sin y cos z, w = aw cos x cos y
  // sin z, aw = -(au + av) (pfield.f:34-78): the modes (+-1, +-1, +-1), of
  // which the kx = 1 half is stored: u = -i au/8, v = -i sgn(ky) av/8,
  // w = -i sgn(kz) aw/8; everything else zero
  const double aw = -(au + av);
  const size_t vs = (size_t)g.xz_tot * n;
  CK(cudaMemsetAsync(c->d_u, 0, c->csz * c->st_elems, c->stream));
  CK(cudaMemsetAsync(c->d_un, 0, c->csz * c->st_elems, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int kc1 = (g.colstart[2] - g.colstart[1] - 1) / 2;
  for (int sz = -1; sz <= 1; sz += 2)
    for (int sy = -1; sy <= 1; sy += 2) {
      const int a = g.colstart[1] + (sz > 0 ? 1 : 2 * kc1);
      const int y = sy > 0 ? 1 : n - 1;
      const double val[3] = {-au / 8., -sy * av / 8., -sz * aw / 8.};   // imaginary parts
      for (int v = 0; v < 3; v++) {
        const size_t o = v * vs + (size_t)a * n + y;
        if (c->prec == PSDNS_PREC_FP64) {
          const double2 e = make_double2(0.0, val[v]);
          CK(cudaMemcpy((double2*)c->d_u + o, &e, sizeof e, cudaMemcpyHostToDevice));
          CK(cudaMemcpy((double2*)c->d_un + o, &e, sizeof e, cudaMemcpyHostToDevice));
        } else {
          const float2 e = make_float2(0.f, (float)val[v]);
          CK(cudaMemcpy((float2*)c->d_u + o, &e, sizeof e, cudaMemcpyHostToDevice));
          CK(cudaMemcpy((float2*)c->d_un + o, &e, sizeof e, cudaMemcpyHostToDevice));
        }
      }
    }
  return 0;
}

int psdns_gpu_particles_set(void* ctx, int64_t np, const double* pos) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (np < 0) return set_error("negative particle count");
  if (np > 0 && c->rk != 2) return set_error("particles are advanced with the RK2 step only");
  if (np > 0 && !pos) return set_error("null positions");
  if (c->d_pos) { cudaFree(c->d_pos); c->d_pos = nullptr; }
  if (c->d_vel) { cudaFree(c->d_vel); c->d_vel = nullptr; }
  c->np = 0;
  if (np == 0) return 0;
  const size_t n3 = (size_t)c->n * c->n * c->n;
  const size_t bsb = n3 * 4 * (c->prec == PSDNS_PREC_FP64 ? sizeof(double) : sizeof(float));
  size_t freeb = 0, totb = 0;
  CK(cudaMemGetInfo(&freeb, &totb));
  const size_t need = (c->d_bs ? 0 : bsb) + sizeof(double) * 6 * (size_t)np;
  if (need + (size_t)256 * 1024 * 1024 > freeb)
    return set_error("particles need %.2f GB of device memory, %.2f GB free", need / 1e9, freeb / 1e9);
  if (!c->d_bs) CK(cudaMalloc(&c->d_bs, bsb));
  CK(cudaMalloc((void**)&c->d_pos, sizeof(double) * 3 * (size_t)np));
  CK(cudaMalloc((void**)&c->d_vel, sizeof(double) * 3 * (size_t)np));
  CK(cudaMemcpy(c->d_pos, pos, sizeof(double) * 3 * (size_t)np, cudaMemcpyHostToDevice));
  CK(cudaMemset(c->d_vel, 0, sizeof(double) * 3 * (size_t)np));
  c->np = np;
  c->part_first = true;
  return 0;
}

int psdns_gpu_particles_init(void* ctx, int64_t nop, int32_t pstart, int32_t kipran) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (pstart != 0 && pstart != -1) return set_error("pstart must be 0 (random) or -1 (lattice)");
  if (c->rk != 2) return set_error("particles are advanced with the RK2 step only");
  if (nop <= 0) return set_error("nop must be positive");
  if (kipran < 1 || kipran > 20) return set_error("kipran must be 1..20 (ranseq.f:131)");
  const long long tot = pstart == -1 ? (long long)nop * nop * nop : nop;
  if (tot > (long long)c->n * c->n * c->n && pstart == -1)
    return set_error("a lattice of %lld particles exceeds the %d^3 grid (partin.f:167)", tot, c->n);
  c->pin_nop = nop;
  c->pin_pstart = pstart;
  c->pin_kipran = kipran;
  return 0;
}

int psdns_gpu_particles_advance(void* ctx, const double* gsh1, double dt_prev) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !gsh1) return set_error("null argument");
  if (c->np == 0 && c->pin_nop == 0) return set_error("no particles");
  if (!c->part_first && !(dt_prev > 0)) return set_error("the particle step needs a positive dt");
  Ops o;
  if (!get_ops(c->prec, c->n, c->nc, o)) return set_error("bad context");
  // the stage-1 shifts and dt that psdns_gpu_step would hold at this point;
  // rk_stage(1) sets both again for its own use
  for (int i = 0; i < 3; i++) c->gsh[i][0] = gsh1[i];
  c->dt = dt_prev;
  if (c->prec == PSDNS_PREC_FP64) fill_shift_tables<double>(*c); else fill_shift_tables<float>(*c);
  if (upload_tables(*c)) return 1;
  if (c->pin_nop > 0 && make_partin(*c)) return 1;
  if (c->np > 0 && o.particles(*c)) return 1;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int psdns_gpu_particles_get(void* ctx, double* pos, double* vel) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (c->np == 0) return set_error("no particles");
  if (pos) CK(cudaMemcpy(pos, c->d_pos, sizeof(double) * 3 * (size_t)c->np, cudaMemcpyDeviceToHost));
  if (vel) CK(cudaMemcpy(vel, c->d_vel, sizeof(double) * 3 * (size_t)c->np, cudaMemcpyDeviceToHost));
  return 0;
}

// hooks/LAG_LOCAL/pop1_file_local.f + pop1_write_local2.f for one writing
// task (nsubset = 1): per group igp = 1..ngp, files <prefix>/<igp>/pvel1g<igp>_s0
// and <prefix>/<igp>/ppos1g<igp>_s0, big-endian unformatted (makefile:251).
// Opened (append = 0) with the record (nopg, nrefp, 4, 3), nopg = 4 nrefp,
// nrefp = np / (1 + 3 ngp); every call appends the record (istep - 1,
// time) and, for each of the three components (velocities u v w, or
// positions x y z), the reference particles pp(1:nrefp) and the three
// satellite sets of the group, pp(nrefp + ((igp-1) 3 + ii - 1) nrefp + 1 :
// ... + nrefp), ii = 1..3 (pop1_write_local2.f:238-262).
int psdns_gpu_particles_write(void* ctx, const char* prefix, int32_t ngp, int32_t istep, int32_t append) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !prefix) return set_error("null argument");
  if (c->np == 0) return set_error("no particles");
  if (ngp < 1 || c->np % (1 + 3 * (long long)ngp) != 0)
    return set_error("particles_write: np = %lld is not nrefp (1 + 3 ngp) for ngp = %d", c->np, ngp);
  const long long nrefp = c->np / (1 + 3 * (long long)ngp);
  if (nrefp > (1LL << 28)) return set_error("particles_write: too many particles for one record");
  std::vector<double> pos(3 * (size_t)c->np), vel(3 * (size_t)c->np);
  if (psdns_gpu_particles_get(c, pos.data(), vel.data())) return 1;
  std::vector<unsigned char> rec;
  for (int igp = 1; igp <= ngp; igp++) {
    for (int kind = 0; kind < 2; kind++) {
      const std::string fn = std::string(prefix) + "/" + std::to_string(igp) + "/" + (kind == 0 ? "pvel" : "ppos") +
                             "1g" + std::to_string(igp) + "_s0";
      FILE* f = std::fopen(fn.c_str(), append ? "ab" : "wb");
      if (!f) return set_error("cannot open %s (the directory %s/%d must exist)", fn.c_str(), prefix, igp);
      bool ok = true;
      if (!append) {
        rec.clear();
        for (uint32_t v : {(uint32_t)(4 * nrefp), (uint32_t)nrefp, 4u, 3u}) be32(rec, v);
        ok = write_record(f, rec.data(), rec.size());
      }
      rec.assign(12, 0);
      rec.clear();
      be32(rec, (uint32_t)(istep - 1));
      rec.resize(12);
      be64(&rec[4], c->time);
      ok = ok && write_record(f, rec.data(), rec.size());
      const double* src = kind == 0 ? vel.data() : pos.data();
      std::vector<unsigned char> row((size_t)8 * nrefp);
      for (int comp = 0; comp < 3 && ok; comp++) {
        const double* a = src + (size_t)comp * c->np;
        for (int set = 0; set < 4 && ok; set++) {
          const long long i0 = set == 0 ? 0 : nrefp + ((long long)(igp - 1) * 3 + set - 1) * nrefp;
          for (long long i = 0; i < nrefp; i++) be64(&row[(size_t)8 * i], a[i0 + i]);
          ok = write_record(f, row.data(), row.size());
        }
      }
      if (std::fclose(f) != 0) ok = false;
      if (!ok) return set_error("write to %s failed", fn.c_str());
    }
  }
  return 0;
}

int psdns_gpu_spectra(void* ctx, int32_t which, double* ek, double* dk, double* eijk, double* stats) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  // the ub work array is free between steps: use it for the sums
  return spectra_of(make_geo(*c), which == PSDNS_FIELD_U ? c->d_u : c->d_un, c->prec, c->p, c->stream, c->d_ub, ek,
                    dk, eijk, stats);
}

int psdns_gpu_gradient_moments(void* ctx, int32_t which, const double* gsh, double* out) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !out) return set_error("null argument");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  Ops o;
  if (!get_ops(c->prec, c->n, c->nc, o)) return set_error("bad context");
  return o.moments(*c, which, gsh, out);
}

int psdns_gpu_transfer_spectrum(void* ctx, const double* gsh, double* tk) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !tk) return set_error("null argument");
  Ops o;
  if (!get_ops(c->prec, c->n, c->nc, o)) return set_error("bad context");
  return o.transfer(*c, gsh, tk);
}

int psdns_gpu_spectra_scales(void* ctx, int32_t which, double* xr, double* yr, double* zr, double* stats) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  return spectra_scales_of(make_geo(*c), which == PSDNS_FIELD_U ? c->d_u : c->d_un, c->prec, c->p, c->stream,
                           c->d_ub, xr, yr, zr, stats);
}

int psdns_gpu_forcing_stats(void* ctx, double* efk, double* eirate, double* erate) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (!(c->p.kforce > 0)) return set_error("context is unforced (kforce = 0)");
  if (efk) for (int k = 0; k < c->kfor; k++) efk[k] = k < (int)c->efk_host.size() ? c->efk_host[k] : 0.0;
  if (eirate) for (int i = 0; i < 3; i++) eirate[i] = c->eirate[i];
  if (erate) *erate = c->erate;
  return 0;
}

int psdns_gpu_forcing_table(void* ctx, double* table, int32_t* kfor, int32_t* k2fo) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (kfor) *kfor = c->kfor;
  if (k2fo) *k2fo = c->k2fo;
  if (table) std::memcpy(table, c->forcing.table.data(), sizeof(double) * c->forcing.table.size());
  return 0;
}

int psdns_gpu_get_stream(void* ctx, void** stream) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !stream) return set_error("null argument");
  *stream = (void*)c->stream;
  return 0;
}

int psdns_gpu_profile(void* ctx, int32_t enable) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  if (enable && !c->ev[0][0][0]) {
    for (int s = 0; s < 4; s++)
      for (int k = 0; k < 6; k++)
        for (int e = 0; e < 2; e++) CK(cudaEventCreate(&c->ev[s][k][e]));
  }
  c->prof = enable != 0;
  for (int k = 0; k < 6; k++) { c->prof_ms[k] = 0; c->prof_n[k] = 0; }
  return 0;
}

int psdns_gpu_kernel_times(void* ctx, double* ms, int64_t* launches) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c) return set_error("null context");
  for (int k = 0; k < 6; k++) {
    if (ms) ms[k] = c->prof_ms[k];
    if (launches) launches[k] = c->prof_n[k];
  }
  return 0;
}

// ---------------------------------------------------------------------------
// learned coarse solver: filter, shell damping, features, correction
// ---------------------------------------------------------------------------
int psdns_gpu_filter_state(const void* fine, void* coarse) {
  const Ctx* f = (const Ctx*)fine;
  Ctx* c = (Ctx*)coarse;
  touch(c);
  if (!f || !c) return set_error("filter_state: null context");
  if (f->prec != c->prec) return set_error("filter_state: both boxes must have the same precision");
  if (!(f->n > c->n)) return set_error("filter_state: the fine box (n = %d) must be larger than the coarse (n = %d)",
                                       f->n, c->n);
  if (f->p.beta1 != c->p.beta1 || f->p.beta2 != c->p.beta2 || f->p.beta3 != c->p.beta3)
    return set_error("filter_state: the boxes must have the same shape (beta)");
  CK(cudaStreamSynchronize(f->stream));
  const size_t tot = 3 * (size_t)c->g.xz_tot * c->n;
  const int blocks = (int)std::min<size_t>((tot + 255) / 256, 148 * 16);
  if (c->prec == PSDNS_PREC_FP64)
    k_filter_state<double><<<blocks, 256, 0, c->stream>>>(make_geo(*f), (const double2*)f->d_un, make_geo(*c),
                                                          (double2*)c->d_u, (double2*)c->d_un);
  else
    k_filter_state<float><<<blocks, 256, 0, c->stream>>>(make_geo(*f), (const float2*)f->d_un, make_geo(*c),
                                                         (float2*)c->d_u, (float2*)c->d_un);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int psdns_gpu_shell_factor(void* ctx, int32_t nshell, const double* f) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !f) return set_error("shell_factor: null argument");
  if (nshell < 1 || nshell >= c->n) return set_error("shell_factor: nshell must be in 1 .. n-1");
  if (!c->d_shf) CK(cudaMalloc((void**)&c->d_shf, sizeof(double) * c->n));
  CK(cudaMemcpyAsync(c->d_shf, f, sizeof(double) * (nshell + 1), cudaMemcpyHostToDevice, c->stream));
  const size_t tot = 3 * (size_t)c->g.xz_tot * c->n;
  const int blocks = (int)std::min<size_t>((tot + 255) / 256, 148 * 16);
  const double b11 = c->p.beta1 * c->p.beta1, b22 = c->p.beta2 * c->p.beta2, b33 = c->p.beta3 * c->p.beta3;
  if (c->prec == PSDNS_PREC_FP64)
    k_shell_factor<double><<<blocks, 256, 0, c->stream>>>(make_geo(*c), (double2*)c->d_u, (double2*)c->d_un,
                                                          c->d_shf, nshell, b11, b22, b33);
  else
    k_shell_factor<float><<<blocks, 256, 0, c->stream>>>(make_geo(*c), (float2*)c->d_u, (float2*)c->d_un, c->d_shf,
                                                         nshell, b11, b22, b33);
  CK(cudaGetLastError());
  // f is borrowed for the call only
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// shells 1 .. K of the coarse box: K = int(kmax + 0.5), kmax = sqrt(2) n / 3
static int resolved_shells(int n) { return (int)(std::sqrt(2.0) * n / 3.0 + 0.5); }

int psdns_gpu_corrector_features(void* ctx, int32_t which, int32_t nshell, float* x) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !x) return set_error("corrector_features: null argument");
  if (nshell < 1 || nshell > resolved_shells(c->n))
    return set_error("corrector_features: nshell must be in 1 .. %d", resolved_shells(c->n));
  std::vector<double> ek(c->n);
  double st[7];
  if (psdns_gpu_spectra(c, which, ek.data(), nullptr, nullptr, st)) return 1;
  // per shell i: i / kmax; the compensated spectrum log10(E(i) i^(5/3) /
  // eps^(2/3)) (clamped to [-10, 10]); the resolution log10(kmax eta),
  // eta = (nu^3 / eps)^(1/4), eps the resolved dissipation (sptr.f:354-365)
  const double kmax = std::sqrt(2.0) * c->n / 3.0, nu = c->p.viscos;
  const double eps = st[1] > 0 ? st[1] : 1e-300;
  const double res = std::log10(kmax * std::pow(nu * nu * nu / eps, 0.25));
  for (int i = 1; i <= nshell; i++) {
    double comp = std::log10(std::max(ek[i], 1e-300) * std::pow((double)i, 5.0 / 3.0) / std::pow(eps, 2.0 / 3.0));
    comp = std::min(10.0, std::max(-10.0, comp));
    x[3 * (i - 1) + 0] = (float)(i / kmax);
    x[3 * (i - 1) + 1] = (float)comp;
    x[3 * (i - 1) + 2] = (float)res;
  }
  return 0;
}

int psdns_gpu_corrector_apply(void* corr, void* ctx, double* info) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!corr || !c) return set_error("corrector_apply: null argument");
  const int K = resolved_shells(c->n);
  std::vector<float> x(3 * K), g(K);
  if (psdns_gpu_corrector_features(c, PSDNS_FIELD_UN, K, x.data())) return 1;
  if (mlp::forward_host(corr, K, x.data(), g.data())) return 1;
  // eddy viscosity nu_t(i) = nu g(i); damping over the last step's dt
  std::vector<double> f(K + 1, 1.0);
  double gmax = 0;
  bool ok = c->dt > 0;
  for (int i = 1; i <= K && ok; i++) {
    const double gi = g[i - 1];
    if (!(gi >= 0) || !(gi < 1e4)) ok = false;   // NaN, negative or runaway: fall back
    gmax = std::max(gmax, gi);
    f[i] = std::exp(-c->p.viscos * gi * (double)i * i * c->dt);
  }
  if (info) {
    info[0] = ok ? 1.0 : 0.0;
    info[1] = gmax;
  }
  if (!ok) return 0;   // the plain solver's step stands
  return psdns_gpu_shell_factor(c, K, f.data());
}

int psdns_gpu_get_time(void* ctx, double* out4) {
  Ctx* c = (Ctx*)ctx;
  touch(c);
  if (!c || !out4) return set_error("null argument");
  out4[0] = c->time;
  out4[1] = c->dt;
  out4[2] = c->velmax;
  out4[3] = (double)c->jstep;
  return 0;
}

}  // extern "C"

// ensembles of boxes (batched stage kernels, CUDA graphs)
#include "ensemble.cuh"
#endif  // PSDNS_INST_N
