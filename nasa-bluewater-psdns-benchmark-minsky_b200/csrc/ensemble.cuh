// ensemble.cuh -- many independent boxes advanced together (included at the
// end of psdns_api.cu, which defines Ctx, Impl and the host helpers; the
// ensemble types and kernel sequences are in ensemble_impl.cuh).

namespace psdns {

static int ens_setup(EnsClass& e) {
#define PSDNS_ECASE(NN)                                                                           \
  case NN:                                                                                        \
    return ens_setup_n<NN>(e);
  switch (e.n) {
    PSDNS_ECASE(16)
    PSDNS_ECASE(32)
    PSDNS_ECASE(48)
    PSDNS_ECASE(64)
    PSDNS_ECASE(96)
    PSDNS_ECASE(128)
    PSDNS_ECASE(256)
    PSDNS_ECASE(512)
    PSDNS_ECASE(1024)
    default:
      return set_error("ensemble: grid size %d not supported", e.n);
  }
#undef PSDNS_ECASE
}

static void ens_free_class(EnsClass* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->graph) cudaGraphDestroy(e->graph);
  void* ptrs[] = {e->d_colstart, e->d_ax, e->d_az, e->d_kymax, e->d_u, e->d_un, e->d_ub,
                  e->d_uz, e->d_tabs, e->d_tw, e->d_normv, e->d_velmax};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (e->h_tabs) cudaFreeHost(e->h_tabs);
  if (e->h_normv) cudaFreeHost(e->h_normv);
  if (e->h_velmax) cudaFreeHost(e->h_velmax);
  if (e->stream) cudaStreamDestroy(e->stream);
  for (Ctx* c : e->box) delete c;
  delete e;
}

static int ens_alloc_class(EnsClass& e) {
  const int n = e.n;
  const bool dbl = e.prec == PSDNS_PREC_FP64;
  const size_t csz = dbl ? sizeof(double2) : sizeof(float2);
  const int tbi = dbl ? Tiles<double>::TB_I : Tiles<float>::TB_I;
  const int tbf = dbl ? Tiles<double>::TB_F : Tiles<float>::TB_F;
  const int tz = dbl ? Tiles<double>::TZ : Tiles<float>::TZ;
  build_geometry(n, e.g);
  e.nzt = n / tz;
  e.nab_i = (e.g.xz_tot + tbi - 1) / tbi;
  e.nab_f = (e.g.xz_tot + tbf - 1) / tbf;
  // per-box strides rounded to 256 bytes so that every box's arrays stay aligned
  auto up = [csz](size_t el) { return ((el * csz + 255) / 256 * 256) / csz; };
  e.st_elems = up((size_t)3 * e.g.xz_tot * n);
  const size_t ubi = dbl ? ubi_var_elems<double>(e.nab_i, n) : ubi_var_elems<float>(e.nab_i, n);
  e.ub_elems = up(std::max((size_t)3 * ubi, (size_t)4 * (dbl ? ubf_var_elems<double>(e.nab_f, n) : ubf_var_elems<float>(e.nab_f, n))));
  e.uz_elems = up((size_t)5 * n * n * e.g.kxn);
  e.tab_bytes = dbl ? TabLayout<double>(n).total : TabLayout<float>(n).total;
  const size_t nb = e.nb;
  size_t freeb = 0, totb = 0;
  CK(cudaMemGetInfo(&freeb, &totb));
  const size_t need = csz * nb * (2 * e.st_elems + e.ub_elems + e.uz_elems);
  if (need + (size_t)256 * 1024 * 1024 > freeb)
    return set_error("ensemble: %d boxes of %d^3 need %.2f GB of device memory, %.2f GB free", e.nb, n,
                     need / 1e9, freeb / 1e9);
  if (ens_setup(e)) return 1;
  CK(cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking));
  CK(cudaMalloc((void**)&e.d_colstart, sizeof(int) * (e.g.kxn + 1)));
  CK(cudaMalloc((void**)&e.d_ax, sizeof(int) * e.g.xz_tot));
  CK(cudaMalloc((void**)&e.d_az, sizeof(int) * e.g.xz_tot));
  CK(cudaMalloc((void**)&e.d_kymax, sizeof(int) * e.g.xz_tot));
  CK(cudaMalloc(&e.d_u, csz * nb * e.st_elems));
  CK(cudaMalloc(&e.d_un, csz * nb * e.st_elems));
  CK(cudaMalloc(&e.d_ub, csz * nb * e.ub_elems));
  CK(cudaMalloc(&e.d_uz, csz * nb * e.uz_elems));
  CK(cudaMalloc(&e.d_tabs, e.tab_bytes * nb));
  CK(cudaMalloc(&e.d_normv, (dbl ? sizeof(double) : sizeof(float)) * nb));
  CK(cudaMalloc((void**)&e.d_velmax, sizeof(unsigned long long) * nb));
  CK(cudaMallocHost(&e.h_tabs, e.tab_bytes * nb));
  CK(cudaMallocHost(&e.h_normv, (dbl ? sizeof(double) : sizeof(float)) * nb));
  CK(cudaMallocHost((void**)&e.h_velmax, sizeof(unsigned long long) * nb));
  std::memset(e.h_tabs, 0, e.tab_bytes * nb);
  std::memset(e.h_normv, 0, (dbl ? sizeof(double) : sizeof(float)) * nb);
  CK(cudaMemcpy(e.d_colstart, e.g.colstart.data(), sizeof(int) * (e.g.kxn + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e.d_ax, e.g.ax.data(), sizeof(int) * e.g.xz_tot, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e.d_az, e.g.az.data(), sizeof(int) * e.g.xz_tot, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e.d_kymax, e.g.kymax.data(), sizeof(int) * e.g.xz_tot, cudaMemcpyHostToDevice));
  CK(cudaMemset(e.d_u, 0, csz * nb * e.st_elems));
  CK(cudaMemset(e.d_un, 0, csz * nb * e.st_elems));
  // each box's host state writes its tables into its slice of the staging block
  for (int b = 0; b < e.nb; b++) {
    Ctx* c = e.box[b];
    c->g = e.g;
    c->n = n;
    c->prec = e.prec;
    c->csz = csz;
    c->h_tabs = (char*)e.h_tabs + (size_t)b * e.tab_bytes;
  }
  return 0;
}

// the device copy of box b's state u (which = 0) or un (which = 1)
static void* ens_state(const EnsClass& e, int b, int which) {
  const size_t csz = e.prec == PSDNS_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  return (char*)(which == PSDNS_FIELD_U ? e.d_u : e.d_un) + (size_t)b * e.st_elems * csz;
}

static void ens_fill_factors(EnsClass& e) {
  for (int b = 0; b < e.nb; b++) {
    Ctx& c = *e.box[b];
    if (e.prec == PSDNS_PREC_FP64) {
      fill_factor_tables<double>(c);
      ((double*)e.h_normv)[b] = c.dt2 / c.n / c.n;
    } else {
      fill_factor_tables<float>(c);
      ((float*)e.h_normv)[b] = (float)(c.dt2 / c.n / c.n);
    }
  }
}

static void ens_fill_shifts(EnsClass& e) {
  for (int b = 0; b < e.nb; b++) {
    Ctx& c = *e.box[b];
    c.jstep += 1;
    draw_shifts(c);
    if (e.prec == PSDNS_PREC_FP64) fill_shift_tables<double>(c); else fill_shift_tables<float>(c);
  }
}

static int ens_upload_tables(EnsClass& e) {
  const size_t rs = e.prec == PSDNS_PREC_FP64 ? sizeof(double) : sizeof(float);
  CK(cudaMemcpyAsync(e.d_tabs, e.h_tabs, e.tab_bytes * e.nb, cudaMemcpyHostToDevice, e.stream));
  CK(cudaMemcpyAsync(e.d_normv, e.h_normv, rs * e.nb, cudaMemcpyHostToDevice, e.stream));
  return 0;
}

// the device part of a fixed-dt step: tables in, both stages, velmax out
static int ens_step_body(EnsClass& e) {
  if (ens_upload_tables(e)) return 1;
  CK(cudaMemsetAsync(e.d_velmax, 0, sizeof(unsigned long long) * e.nb, e.stream));
  const int sub = e.sub > 0 ? e.sub : e.nb;
  for (int b0 = 0; b0 < e.nb; b0 += sub) {
    const int m = std::min(sub, e.nb - b0);
    if (e.stage_a(e, 1, b0, m) || e.stage_b(e, 1, b0, m) || e.stage_a(e, 2, b0, m) || e.stage_b(e, 2, b0, m))
      return 1;
  }
  CK(cudaMemcpyAsync(e.h_velmax, e.d_velmax, sizeof(unsigned long long) * e.nb, cudaMemcpyDeviceToHost, e.stream));
  return 0;
}

static int ens_read_velmax(EnsClass& e) {
  for (int b = 0; b < e.nb; b++) {
    double vm;
    std::memcpy(&vm, e.h_velmax + b, sizeof vm);
    e.box[b]->velmax = vm;
  }
  return 0;
}

// one step of every box of a class with a fixed dt: the first one runs
// eagerly and is captured, later ones replay the graph
static int ens_step_fixed(EnsClass& e) {
  ens_fill_shifts(e);
  // dt, time and dt2 of the step (step.f:247-262); the Courant check needs
  // this step's velmax and is made after the step
  for (Ctx* c : e.box) step_control(*c);
  if (!e.tuned) {
    // tuning steps (real steps: the sub-batch size and the tiles change no
    // result), timed with events on the class stream
    if (e.cands.empty()) {
      if (e.phase == 0) {
        for (int s = e.nb; s >= 1; s /= 2) e.cands.push_back({s, 0, 0});
        ens_fill_factors(e);   // dt is fixed: the factor tables never change
      } else {
        for (int v = 0; v < 3; v++)
          e.cands.push_back(e.phase == 1 ? EnsClass::Cand{e.sub, v, e.k4v} : EnsClass::Cand{e.sub, e.k2v, v});
      }
      e.cand_ms.assign(e.cands.size(), 1e30f);
      e.trial = 0;
      e.rep = 0;
    }
    const EnsClass::Cand cd = e.cands[e.trial];
    e.sub = cd.sub;
    e.k2v = cd.k2v;
    e.k4v = cd.k4v;
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, e.stream));
    const int rc = ens_step_body(e);
    CK(cudaEventRecord(t1, e.stream));
    CK(cudaEventSynchronize(t1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return 1;
    e.cand_ms[e.trial] = std::min(e.cand_ms[e.trial], ms);
    if (++e.rep == 2) {
      e.rep = 0;
      e.trial += 1;
    }
    if (e.trial == (int)e.cands.size()) {
      int best = 0;
      for (size_t i = 1; i < e.cands.size(); i++)
        if (e.cand_ms[i] < e.cand_ms[best]) best = (int)i;
      if (e.phase == 0) e.default_ms = e.cand_ms[0];
      e.best_ms = e.cand_ms[best];
      e.sub = e.cands[best].sub;
      e.k2v = e.cands[best].k2v;
      e.k4v = e.cands[best].k4v;
      e.cands.clear();
      e.phase += 1;
      if (!e.tile_tune || e.phase == 3) e.tuned = true;
    }
    return 0;
  }
  if (!e.gexec) {
    CK(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
    const int rc = ens_step_body(e);
    cudaGraph_t gr = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e.stream, &gr);
    if (rc) { if (gr) cudaGraphDestroy(gr); return 1; }
    if (ce != cudaSuccess) return set_error("graph capture failed: %s", cudaGetErrorString(ce));
    e.graph = gr;
    CK(cudaGraphInstantiate(&e.gexec, e.graph, 0));
  }
  CK(cudaGraphLaunch(e.gexec, e.stream));
  return 0;
}

}  // namespace psdns

extern "C" {

int psdns_gpu_ensemble_create(const psdns_params* p, int32_t count, void** out) {
  if (!p || !out) return set_error("null argument");
  *out = nullptr;
  if (count <= 0) return set_error("ensemble needs at least one box");
  const int prec = p[0].precision;
  for (int i = 0; i < count; i++) {
    const psdns_params& q = p[i];
    if (q.nx != q.ny || q.nx != q.nz) return set_error("box %d: only cubic boxes are supported", i);
    if (q.precision != prec) return set_error("box %d: all boxes of an ensemble share one precision", i);
    if (q.precision != PSDNS_PREC_FP32 && q.precision != PSDNS_PREC_FP64) return set_error("box %d: precision", i);
    if (q.nc != 0) return set_error("box %d: ensembles carry no passive scalar (nc = 0)", i);
    if (q.kforce > 0) return set_error("box %d: ensembles are unforced (kforce = 0)", i);
    if (q.rkmethod == 4 || q.dft != PSDNS_DFT_FP32)
      return set_error("box %d: ensembles run the RK2 step with the FP32 transforms", i);
    if (q.kshift < 1 || q.kshift > 4) return set_error("box %d: kshift must be 1..4", i);
    if (q.ksran < 1 || q.ksran > 20) return set_error("box %d: RNG sequence must be 1..20", i);
    if (q.seed_input <= 0) return set_error("box %d: seed must be positive", i);
    if (q.cfl <= 0. && !(q.dt > 0.)) return set_error("box %d: fixed dt must be positive when cfl <= 0", i);
    if (q.beta1 != p[0].beta1 || q.beta2 != p[0].beta2 || q.beta3 != p[0].beta3)
      return set_error("box %d: all boxes share beta", i);
  }
  Ensemble* en = new Ensemble();
  en->count = count;
  en->prec = prec;
  en->where.resize(count);
  // group boxes by n, in order of first appearance
  for (int i = 0; i < count; i++) {
    int k = -1;
    for (size_t j = 0; j < en->cls.size(); j++)
      if (en->cls[j]->n == p[i].nx) k = (int)j;
    if (k < 0) {
      EnsClass* e = new EnsClass();
      e->n = p[i].nx;
      e->prec = prec;
      en->cls.push_back(e);
      k = (int)en->cls.size() - 1;
    }
    EnsClass* e = en->cls[k];
    Ctx* c = new Ctx();
    c->p = p[i];
    c->rng.init(p[i].seed_input);
    c->dt0 = p[i].dt;
    c->dt = p[i].dt;
    e->box.push_back(c);
    e->index.push_back(i);
    if (p[i].cfl > 0.) e->fixed_dt = false;
    en->where[i] = {k, e->nb};
    e->nb += 1;
  }
  for (EnsClass* e : en->cls) {
    if (ens_alloc_class(*e)) {
      psdns_gpu_ensemble_destroy(en);
      return 1;
    }
  }
  *out = en;
  return 0;
}

int psdns_gpu_ensemble_destroy(void* ens) {
  Ensemble* en = (Ensemble*)ens;
  if (!en) return 0;
  for (EnsClass* e : en->cls) ens_free_class(e);
  delete en;
  return 0;
}

int psdns_gpu_ensemble_field_init(void* ens, const int32_t* seeds) {
  Ensemble* en = (Ensemble*)ens;
  if (!en || !seeds) return set_error("null argument");
  for (int i = 0; i < en->count; i++)
    if (seeds[i] <= 0) return set_error("box %d: seed %d must be positive", i, seeds[i]);
  for (EnsClass* e : en->cls) {
    const Geometry& g = e->g;
    const int n = e->n;
    std::vector<long long> off(g.xz_tot);
    long long acc = 0;
    for (int a = 0; a < g.xz_tot; a++) {
      off[a] = acc;
      const int km = std::min(g.kymax[a], n / 2 - 1);
      long long cnt = km >= 0 ? 2LL * km + 1 : 0;
      if (a == 0 && cnt > 0) cnt -= 1;
      acc += cnt;
    }
    long long* d_off = nullptr;
    CK(cudaMalloc(&d_off, sizeof(long long) * g.xz_tot));
    cudaError_t err = cudaMemcpy(d_off, off.data(), sizeof(long long) * g.xz_tot, cudaMemcpyHostToDevice);
    const Geo geo = ens_geo(*e);
    const int kc0 = n / 2 - 1 - g.cut[0];
    for (int b = 0; b < e->nb && err == cudaSuccess; b++) {
      const psdns_params& q = e->box[b]->p;
      const uint32_t seed = (uint32_t)seeds[e->index[b]];
      if (e->prec == PSDNS_PREC_FP64) {
        double2* un = (double2*)ens_state(*e, b, PSDNS_FIELD_UN);
        double2* u = (double2*)ens_state(*e, b, PSDNS_FIELD_U);
        k_field_init<double><<<148 * 8, 256, 0, e->stream>>>(geo, d_off, seed, q.beta1, q.beta2, q.beta3, un, u);
        k_field_consym<double><<<148, 256, 0, e->stream>>>(n, kc0, g.xz_tot, un, u);
      } else {
        float2* un = (float2*)ens_state(*e, b, PSDNS_FIELD_UN);
        float2* u = (float2*)ens_state(*e, b, PSDNS_FIELD_U);
        k_field_init<float><<<148 * 8, 256, 0, e->stream>>>(geo, d_off, seed, q.beta1, q.beta2, q.beta3, un, u);
        k_field_consym<float><<<148, 256, 0, e->stream>>>(n, kc0, g.xz_tot, un, u);
      }
      err = cudaGetLastError();
    }
    const cudaError_t e2 = cudaStreamSynchronize(e->stream);
    cudaFree(d_off);
    if (err != cudaSuccess || e2 != cudaSuccess)
      return set_error("ensemble field init failed: %s", cudaGetErrorString(err != cudaSuccess ? err : e2));
  }
  return 0;
}

int psdns_gpu_ensemble_set_state(void* ens, int32_t box, const double* un, int32_t layout) {
  Ensemble* en = (Ensemble*)ens;
  if (!en || !un) return set_error("null argument");
  if (box < 0 || box >= en->count) return set_error("box %d out of range", box);
  if (layout != PSDNS_LAYOUT_YCYL) return set_error("ensemble state I/O uses PSDNS_LAYOUT_YCYL");
  EnsClass& e = *en->cls[en->where[box].first];
  const int b = en->where[box].second;
  const size_t vs = (size_t)e.g.xz_tot * e.n;
  for (int v = 0; v < 3; v++) {
    CK(cudaMemcpyAsync(e.d_ub, un + 2 * v * vs, sizeof(double2) * vs, cudaMemcpyHostToDevice, e.stream));
    if (e.prec == PSDNS_PREC_FP64)
      k_from_f64<double><<<148 * 8, 256, 0, e.stream>>>((const double2*)e.d_ub,
                                                         (double2*)ens_state(e, b, PSDNS_FIELD_UN) + v * vs,
                                                         (double2*)ens_state(e, b, PSDNS_FIELD_U) + v * vs, vs);
    else
      k_from_f64<float><<<148 * 8, 256, 0, e.stream>>>((const double2*)e.d_ub,
                                                        (float2*)ens_state(e, b, PSDNS_FIELD_UN) + v * vs,
                                                        (float2*)ens_state(e, b, PSDNS_FIELD_U) + v * vs, vs);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(e.stream));
  return 0;
}

int psdns_gpu_ensemble_get_state(void* ens, int32_t box, double* out, int32_t which, int32_t layout) {
  Ensemble* en = (Ensemble*)ens;
  if (!en || !out) return set_error("null argument");
  if (box < 0 || box >= en->count) return set_error("box %d out of range", box);
  if (layout != PSDNS_LAYOUT_YCYL) return set_error("ensemble state I/O uses PSDNS_LAYOUT_YCYL");
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  EnsClass& e = *en->cls[en->where[box].first];
  const int b = en->where[box].second;
  const size_t vs = (size_t)e.g.xz_tot * e.n;
  for (int v = 0; v < 3; v++) {
    if (e.prec == PSDNS_PREC_FP64)
      k_to_f64<double><<<148 * 8, 256, 0, e.stream>>>((const double2*)ens_state(e, b, which) + v * vs,
                                                       (double2*)e.d_ub, vs);
    else
      k_to_f64<float><<<148 * 8, 256, 0, e.stream>>>((const float2*)ens_state(e, b, which) + v * vs,
                                                      (double2*)e.d_ub, vs);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out + 2 * v * vs, e.d_ub, sizeof(double2) * vs, cudaMemcpyDeviceToHost, e.stream));
  }
  CK(cudaStreamSynchronize(e.stream));
  return 0;
}

int psdns_gpu_ensemble_tuning(void* ens, int32_t cap, double* out, int32_t* nclasses) {
  Ensemble* E = (Ensemble*)ens;
  if (!E || !nclasses) return set_error("null argument");
  *nclasses = (int32_t)E->cls.size();
  for (size_t i = 0; i < E->cls.size() && (int32_t)i < cap && out; i++) {
    const EnsClass& e = *E->cls[i];
    const int xt2 = e.prec == PSDNS_PREC_FP64 ? Tiles<double>::XT2 : Tiles<float>::XT2;
    const int xt4 = k4_xt(e.prec == PSDNS_PREC_FP64, e.n);
    const int m[3][2] = {{1, 1}, {1, 2}, {2, 1}};   // tile factor of variant 0, 1, 2: num/den
    double* r = out + 8 * i;
    r[0] = e.n;
    r[1] = e.nb;
    r[2] = e.tuned ? 1 : 0;
    r[3] = e.sub > 0 ? e.sub : e.nb;
    r[4] = xt2 * m[e.k2v][0] / m[e.k2v][1];
    r[5] = xt4 * m[e.k4v][0] / m[e.k4v][1];
    r[6] = e.default_ms;
    r[7] = e.best_ms;
  }
  return 0;
}

int psdns_gpu_ensemble_step(void* ens, int32_t nsteps, double* info) {
  Ensemble* en = (Ensemble*)ens;
  if (!en) return set_error("null ensemble");
  if (nsteps < 0) return set_error("negative step count");
  int status = 0;
  for (int s = 0; s < nsteps; s++) {
    // fixed-dt classes: one graph launch each, all classes in flight together
    for (EnsClass* e : en->cls)
      if (e->fixed_dt && ens_step_fixed(*e)) return 1;
    // adaptive classes: stage-1 part A of every class, then dt from velmax
    for (EnsClass* e : en->cls) {
      if (e->fixed_dt) continue;
      ens_fill_shifts(*e);
      if (ens_upload_tables(*e)) return 1;
      CK(cudaMemsetAsync(e->d_velmax, 0, sizeof(unsigned long long) * e->nb, e->stream));
      if (e->stage_a(*e, 1, 0, e->nb)) return 1;
      CK(cudaMemcpyAsync(e->h_velmax, e->d_velmax, sizeof(unsigned long long) * e->nb, cudaMemcpyDeviceToHost,
                         e->stream));
    }
    for (EnsClass* e : en->cls) {
      if (e->fixed_dt) continue;
      CK(cudaStreamSynchronize(e->stream));
      ens_read_velmax(*e);
      for (Ctx* c : e->box)
        if (step_control(*c)) status = 2;
      ens_fill_factors(*e);
      if (ens_upload_tables(*e)) return 1;
      if (e->stage_b(*e, 1, 0, e->nb) || e->stage_a(*e, 2, 0, e->nb) || e->stage_b(*e, 2, 0, e->nb)) return 1;
    }
    // the pinned tables are refilled next step: wait for every class
    for (EnsClass* e : en->cls) {
      CK(cudaStreamSynchronize(e->stream));
      if (!e->fixed_dt) continue;
      ens_read_velmax(*e);
      for (Ctx* c : e->box) {
        const double cn = c->velmax * c->dt / 2. / (4. * std::atan(1.));
        if (c->p.cfl < 0. && cn > 1) {
          set_error("courant number %.4f exceeds 1 (step.f:292)", cn);
          status = 2;
        }
      }
    }
  }
  if (info) {
    const double pi = 4. * std::atan(1.);
    for (EnsClass* e : en->cls)
      for (int b = 0; b < e->nb; b++) {
        const Ctx& c = *e->box[b];
        double* o = info + 8 * (size_t)e->index[b];
        o[0] = c.dt; o[1] = c.time; o[2] = c.velmax; o[3] = c.velmax * c.dt / 2. / pi;
        o[4] = c.gsh[0][0]; o[5] = c.gsh[1][0]; o[6] = c.gsh[2][0]; o[7] = (double)c.jstep;
      }
  }
  return status;
}

int psdns_gpu_ensemble_spectra(void* ens, int32_t box, int32_t which, double* ek, double* dk, double* eijk,
                               double* stats) {
  Ensemble* en = (Ensemble*)ens;
  if (!en) return set_error("null ensemble");
  if (box < 0 || box >= en->count) return set_error("box %d out of range", box);
  if (which != PSDNS_FIELD_U && which != PSDNS_FIELD_UN) return set_error("which must be U or UN");
  EnsClass& e = *en->cls[en->where[box].first];
  const int b = en->where[box].second;
  return spectra_of(ens_geo(e), ens_state(e, b, which), e.prec, e.box[b]->p, e.stream, e.d_ub, ek, dk, eijk,
                    stats);
}

}  // extern "C"
