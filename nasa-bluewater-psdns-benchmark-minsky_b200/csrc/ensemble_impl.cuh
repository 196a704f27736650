// ensemble_impl.cuh -- types and kernel sequences of ensembles (included by
// psdns_api.cu after Impl; the host side is ensemble.cuh).
//
// Boxes of the same grid size n form a class: their states, work arrays and
// stage tables are stored back to back, and every stage kernel runs once per
// class with the box as an extra grid dimension (Geo::sbox/bbox/zbox,
// StageTables::tbox/normv).  A step therefore costs ten kernel launches per
// distinct n, whatever the number of boxes.  Each box keeps the host state
// of a single-box run (its own shift RNG stream, dt, time), so box b of an
// ensemble follows exactly the run of a single context with the same
// parameters.  Classes whose boxes all use a fixed dt (cfl <= 0) replay each
// step from a captured CUDA graph; with cfl > 0 the host reads the classes'
// velmax once per step, between stage-1 parts A and B, to set every box's dt.

namespace psdns {

struct EnsClass {
  int n = 0, nb = 0, prec = 0;
  std::vector<Ctx*> box;          // host state per box (no device arrays of its own)
  std::vector<int> index;         // ensemble index of each box
  Geometry g;
  int nzt = 0, nab_i = 0, nab_f = 0;
  size_t st_elems = 0, ub_elems = 0, uz_elems = 0, tab_bytes = 0;
  int *d_colstart = nullptr, *d_ax = nullptr, *d_az = nullptr, *d_kymax = nullptr;
  void *d_u = nullptr, *d_un = nullptr, *d_ub = nullptr, *d_uz = nullptr, *d_tabs = nullptr, *d_tw = nullptr;
  void* d_normv = nullptr;
  unsigned long long* d_velmax = nullptr;
  void *h_tabs = nullptr, *h_normv = nullptr;
  unsigned long long* h_velmax = nullptr;
  cudaStream_t stream = nullptr;
  bool fixed_dt = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int (*stage_a)(EnsClass&, int, int, int) = nullptr;
  int (*stage_b)(EnsClass&, int, int, int) = nullptr;
  // boxes per launch of the fixed-dt step (0: all).  A sub-batch runs its
  // whole step (both stages) before the next starts, so that its work
  // arrays can stay in the 126 MB L2; the first steps try candidate sizes
  // (they are real steps: the batching does not change any result) and the
  // fastest is kept for the captured graph.
  int sub = 0;
  bool tuned = false;
  // the tuner also chooses the FFT tiles of K2 and K4 (x lines per block:
  // variant 0 = Tiles<T>, 1 = half, 2 = double; boxes of n <= 128 only).
  // Phases: 0 sub-batch size, 1 K2 tile, 2 K4 tile; every candidate runs
  // two real steps and keeps the faster (the first also loads its kernels).
  int k2v = 0, k4v = 0;
  bool tile_tune = false;   // n <= 128
  int phase = 0, trial = 0, rep = 0;
  struct Cand { int sub, k2v, k4v; };
  std::vector<Cand> cands;
  std::vector<float> cand_ms;
  float default_ms = 0.f, best_ms = 0.f;   // the first candidate (all defaults) and the choice
};

struct Ensemble {
  int count = 0, prec = 0;
  std::vector<EnsClass*> cls;
  std::vector<std::pair<int, int>> where;   // box -> (class, slot)
};

static Geo ens_geo(const EnsClass& e) {
  Geo g;
  g.n = e.n; g.kxn = e.g.kxn; g.xz_tot = e.g.xz_tot; g.nzt = e.nzt;
  g.nab_i = e.nab_i; g.nab_f = e.nab_f;
  g.colstart = e.d_colstart; g.ax = e.d_ax; g.az = e.d_az; g.kymax = e.d_kymax;
  g.sbox = e.st_elems; g.bbox = e.ub_elems; g.zbox = e.uz_elems;
  return g;
}

template <typename T>
static StageTables<T> ens_tables(const EnsClass& e, int ks, int b0) {
  TabLayout<T> L(e.n);
  const char* b = (const char*)e.d_tabs + (size_t)b0 * e.tab_bytes;
  const psdns_params& p = e.box[0]->p;
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
  st.forc = nullptr;
  st.kfor = 0; st.k2fo = 0; st.kforce2 = 0;
  st.b11 = (T)(p.beta1 * p.beta1);
  st.b22 = (T)(p.beta2 * p.beta2);
  st.b33 = (T)(p.beta3 * p.beta3);
  st.norm = T(0);
  st.spf = nullptr;
  st.tbox = e.tab_bytes;
  st.normv = (const T*)e.d_normv + b0;
  return st;
}

template <typename T, int N> struct EnsImpl {
  using C = C2<T>;
  using TL = Tiles<T>;
  using I = Impl<T, N, 0>;
  // tile variants of K2 and K4 are instantiated for small boxes only
  static constexpr bool kTiles = N <= 128;

  // K2 / K4 with XT x lines per block (0: the default tile)
  template <int XT>
  static void k2(EnsClass& e, const Geo& g, const C* ub, C* uz, const C* tw, const StageTables<T>& st, int nb) {
    if constexpr (XT == 0 || kTiles) {
      constexpr int X = XT > 0 ? XT : TL::XT2;
      k_zinv<T, N, 0, false, false, XT><<<dim3(N, (e.g.kxn + X - 1) / X, 3 * nb), Launch<T, N, X>::THREADS,
                                          I::TWB + sizeof(C) * X * I::L, e.stream>>>(g, ub, uz, tw, st.b11, st.b33);
    }
  }
  template <int XT>
  static void k4(EnsClass& e, const Geo& g, const C* uz, C* ub, const C* tw, const StageTables<T>& st, int nb) {
    if constexpr (XT == 0 || kTiles) {
      constexpr int X = XT > 0 ? XT : k4_xt(sizeof(T) == 8, N);
      k_zfwd<T, N, 0, false, XT><<<dim3(N / TL::YT4, (e.g.kxn + X - 1) / X, nb), K4LaunchX<T, N, X>::THREADS,
                                   K4LaunchX<T, N, X>::SMEM, e.stream>>>(g, uz, ub, tw, st.b11, st.b33);
    }
  }

  // boxes b0 .. b0 + nb - 1
  static int stage_a(EnsClass& e, int kstep, int b0, int nb) {
    const Geo g = ens_geo(e);
    const StageTables<T> st = ens_tables<T>(e, kstep - 1, b0);
    const C* tw = (const C*)e.d_tw;
    C* u = (C*)e.d_u + (size_t)b0 * e.st_elems;
    C* ub = (C*)e.d_ub + (size_t)b0 * e.ub_elems;
    C* uz = (C*)e.d_uz + (size_t)b0 * e.uz_elems;
    const int kxn = e.g.kxn;
    k_yinv<T, N><<<dim3(k1_blocks<T>(e.nab_i), 3, nb), K1Launch<T, N>::THREADS, I::sm1(), e.stream>>>(g, st, u, ub, tw);
    switch (kTiles ? e.k2v : 0) {
      case 1: k2<TL::XT2 / 2>(e, g, ub, uz, tw, st, nb); break;
      case 2: k2<TL::XT2 * 2>(e, g, ub, uz, tw, st, nb); break;
      default: k2<0>(e, g, ub, uz, tw, st, nb);
    }
    k_xchain<T, N><<<dim3(e.nzt, N, nb), K3Launch<T, N, 0>::THREADS, I::sm3(), e.stream>>>(
        g, uz, tw, st.b11, st.b22, st.b33, e.d_velmax + b0, kstep == 1 ? 1 : 0);
    switch (kTiles ? e.k4v : 0) {
      case 1: k4<k4_xt(sizeof(T) == 8, N) / 2>(e, g, uz, ub, tw, st, nb); break;
      case 2: k4<k4_xt(sizeof(T) == 8, N) * 2>(e, g, uz, ub, tw, st, nb); break;
      default: k4<0>(e, g, uz, ub, tw, st, nb);
    }
    CK(cudaGetLastError());
    return 0;
  }

  static int stage_b(EnsClass& e, int kstep, int b0, int nb) {
    const Geo g = ens_geo(e);
    const StageTables<T> st = ens_tables<T>(e, kstep - 1, b0);
    constexpr int TH = K5Launch<T, N, 0>::THREADS;
    const C* ub = (const C*)e.d_ub + (size_t)b0 * e.ub_elems;
    C* u = (C*)e.d_u + (size_t)b0 * e.st_elems;
    C* un = (C*)e.d_un + (size_t)b0 * e.st_elems;
    if (kstep == 1)
      k_yfwd<T, N, 1><<<dim3(e.nab_f, nb), TH, I::sm5(), e.stream>>>(g, st, ub, u, un, (const C*)e.d_tw, nullptr);
    else
      k_yfwd<T, N, 2><<<dim3(e.nab_f, nb), TH, I::sm5(), e.stream>>>(g, st, ub, u, un, (const C*)e.d_tw, nullptr);
    CK(cudaGetLastError());
    return 0;
  }

  static int setup(EnsClass& e) {
    if (I::setup()) return 1;
    Ctx tmp;
    if (I::twiddles(tmp)) return 1;
    e.d_tw = tmp.d_tw;
    e.stage_a = &EnsImpl::stage_a;
    e.stage_b = &EnsImpl::stage_b;
    e.tile_tune = kTiles;
    return 0;
  }
};

template <int N> int ens_setup_n(EnsClass& e) {
  return e.prec == PSDNS_PREC_FP64 ? EnsImpl<double, N>::setup(e) : EnsImpl<float, N>::setup(e);
}

}  // namespace psdns
