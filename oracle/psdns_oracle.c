/*
 * psdns_oracle.c -- CPU FP64 restatement of the PSDNS RK2 time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, as the checker.
 *
 * Parity status: pinned only by the reference's own shipped checks, otherwise
 * UNPINNED at the FFT boundary.  The reference (a Fortran/MPI code, PSDNS)
 * builds against FFTW 3, which is neither vendored nor pinned in the reference
 * tree, and it ships no golden vectors; its only correctness checks are the
 * eulstat criteria of its example runs (README.spp:101-105, the sinusoidal
 * field of hooks/initial_conditions/pfield.f) and pcheck.f's exact values of
 * that field on the grid, which tests/test_reference_criteria.py applies to
 * this restatement.  The reference cannot be compiled in this container (no
 * Fortran compiler, MPI or FFTW).  This restatement therefore follows the
 * reference's arithmetic statement by statement (citations below, paths
 * relative to the PSDNS project) and uses its own FP64 FFT, which tests
 * cross-check against numpy.fft.
 *
 * Storage follows the reference's own single-rank layout:
 *   y-cylinders  uy(ny, num_al, nv)   -> here u[v][a][y]   (complex)
 *   z-pencils    uz(nz, xisz, yjsz)   -> here z[v][y][x][z] (complex, x < kxn)
 *   x-pencils    ux(nx, zisz, yjsz)   -> here p[v][y][z][x] (real)
 * where a enumerates the (kx,kz) columns of the cylinder in the order of
 * next_xz (mpisetup.f:710-732).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cx;

static inline cx cmul(cx a, cx b) { cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cx cadd(cx a, cx b) { cx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cx csub(cx a, cx b) { cx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cx cscale(double s, cx a) { cx r = {s * a.re, s * a.im}; return r; }
static inline cx cconj(cx a) { cx r = {a.re, -a.im}; return r; }
static inline cx cmk(double re, double im) { cx r = {re, im}; return r; }
static const cx CZERO = {0.0, 0.0};

/* ------------------------------------------------------------------------ */
/* Random numbers: ranu.f:22-30 (32-bit multiplicative LCG, multiplier      */
/* 65539) with the sequence bookkeeping of ranseq.f:58-141 (20 sequences,  */
/* all seeded with seed_input).                                             */
/* ------------------------------------------------------------------------ */
typedef struct {
    int32_t iseq[20];
    int klast;      /* 1-based */
    int32_t iseed;
    int ifst;
    int32_t seed_input;
} orc_rng;

static void rng_init(orc_rng *r, int32_t seed_input)
{
    memset(r, 0, sizeof(*r));
    r->seed_input = seed_input;
}

/* ranseq(k,0), ranseq.f:62-141 (k > 0 only) */
static void rng_ranseq(orc_rng *r, int k)
{
    if (r->ifst == 0) {
        r->ifst = 1;
        for (int i = 0; i < 20; i++) r->iseq[i] = r->seed_input;
        r->klast = 1;
        r->iseed = r->iseq[0];
    }
    r->iseq[r->klast - 1] = r->iseed;
    r->klast = k;
    r->iseed = r->iseq[k - 1];
}

/* ranu, ranu.f:27-29: iseed*65539 with 32-bit wrap, folded to >= 0 */
static double rng_ranu(orc_rng *r)
{
    uint32_t s = (uint32_t)r->iseed * 65539u;
    int32_t is = (int32_t)s;
    if (is < 0) is = (int32_t)((uint32_t)is + 2147483647u + 1u);
    r->iseed = is;
    return (double)is * 0.46566127e-9;
}

/* ------------------------------------------------------------------------ */
/* FP64 FFT (own implementation; mixed radix 2/3/5 with a direct-DFT        */
/* fallback).  Unnormalised, X_k = sum_j x_j exp(sign*2*pi*i*j*k/n).        */
/* ------------------------------------------------------------------------ */
typedef struct { int n; cx *w; } fft_tw;   /* w[m] = exp(-2 pi i m / n) */

static void tw_make(fft_tw *t, int n)
{
    t->n = n;
    t->w = (cx *)malloc(sizeof(cx) * (size_t)n);
    for (int m = 0; m < n; m++) {
        /* reduce the angle to keep full FP64 accuracy */
        double ang = -2.0 * M_PI * (double)m / (double)n;
        t->w[m] = cmk(cos(ang), sin(ang));
    }
}

static void fft_rec(cx *x, cx *tmp, int n, int stride_tw, const fft_tw *t)
{
    if (n == 1) return;
    int p = 0;
    if (n % 4 == 0) p = 4; else if (n % 2 == 0) p = 2; else if (n % 3 == 0) p = 3; else if (n % 5 == 0) p = 5;
    if (p == 0) { /* direct DFT for other primes */
        for (int k = 0; k < n; k++) {
            cx s = CZERO;
            for (int j = 0; j < n; j++) {
                long idx = ((long)j * k) % n;
                s = cadd(s, cmul(x[j], t->w[idx * stride_tw]));
            }
            tmp[k] = s;
        }
        memcpy(x, tmp, sizeof(cx) * (size_t)n);
        return;
    }
    int m = n / p;
    /* decimation in time: split into p interleaved subsequences */
    for (int r = 0; r < p; r++)
        for (int j = 0; j < m; j++) tmp[r * m + j] = x[j * p + r];
    for (int r = 0; r < p; r++) fft_rec(tmp + r * m, x + r * m, m, stride_tw * p, t);
    for (int k = 0; k < m; k++) {
        cx v[5];
        for (int r = 0; r < p; r++) {
            v[r] = tmp[r * m + k];
            if (r) v[r] = cmul(v[r], t->w[(long)r * k * stride_tw]);
        }
        for (int q = 0; q < p; q++) {
            cx s = CZERO;
            for (int r = 0; r < p; r++) {
                long e = ((long)r * q * m) % n;   /* W_p^{rq} = W_n^{rqm} */
                s = cadd(s, r == 0 ? v[0] : cmul(v[r], t->w[e * stride_tw]));
            }
            x[q * m + k] = s;
        }
    }
}

/* forward (sign=-1) or backward (sign=+1) unnormalised complex FFT */
static void fft_line(cx *x, cx *tmp, int n, int sign, const fft_tw *t)
{
    if (sign > 0) for (int j = 0; j < n; j++) x[j].im = -x[j].im;
    fft_rec(x, tmp, n, 1, t);
    if (sign > 0) for (int j = 0; j < n; j++) x[j].im = -x[j].im;
}

void orc_fft(double *x, int n, int sign)
{
    fft_tw t; tw_make(&t, n);
    cx *tmp = (cx *)malloc(sizeof(cx) * (size_t)n);
    fft_line((cx *)x, tmp, n, sign, &t);
    free(tmp); free(t.w);
}

/* ------------------------------------------------------------------------ */
/* Context                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n, kxn, xz_tot;
    int *cut;       /* cut_z(x), mpisetup.f:322-332 */
    int *kc;        /* largest |kz| kept in column x */
    int *colstart;  /* first a of column x */
    int *ax, *az;   /* per a: x index (0-based), z index (0-based, 0..n-1) */
    int *kymax;     /* per a: largest |ky| inside the sphere, masks.f:67-77 */
    double *kx, *ky, *kz;  /* init.f:15-27 */
    double b11, b22, b33;  /* init.f:33-37 (beta^2) */
    double viscos, cfl, dt0, dt, dt2, time, velmax;
    int kshift, ksran;
    int nc;                /* passive scalars: 0 or 1 */
    double beta[3];        /* init.f:33-37 */
    double pr, cb[3];      /* Schmidt number; cb = beta * grad (init.f:42-45) */
    double *xdif, *ydif, *zdif;  /* step.f:387-407 */
    orc_rng rng;
    double gsh[3][2];      /* shifts.f */
    double gsh4[3][2];     /* gsh(:,3:4) drawn by the RKFOUR-compiled build */
    int jstep;
    cx *sx, *sy, *sz;      /* [2][n]: shifts.f:146-178 */
    double *xfac, *yfac, *zfac;  /* step.f:366-385 */
    cx *u, *un;            /* [3+nc][xz_tot][n] */
    fft_tw tw;
    int status;
    /* Eswaran-Pope forcing (force.f, vfuo.f, vfiuo.f, raniuo.f, rann2.f) */
    double kforce, tforce, epsfor, tfiuo;
    int kranf1, kranf2, kfor, k2fo, nrproc, ffirst;
    double t1, t2, siga;
    double *suo, *svo, *velinc, *w1, *w2;
    cx *forc;              /* for(kfor,k2fo,k2fo,3) */
    double *efkz;          /* efkz(k,i), k = 1..kfor */
    double g_tab[202], g_dtab[202], g_p1;
    int g_ready;
    /* particles: pp(np,1:3) positions, pp(np,4:6) velocities (column-major) */
    long np;
    double *pp;            /* [9][np] */
    int part_first;
    long pin_nop;          /* partin request pending at the first particle phase */
    int pin_pstart, pin_kipran;
    /* timestep_module.f:295-308: rkmethod 2 (proc4a/proc4b) or 4
     * (advanc_1..4 with the accumulator u1 of comp_set.f:72) */
    int rkmethod;
    cx *u1;
} orc_ctx;

static int mask_ok(const orc_ctx *c, int a, int y)
{
    int n = c->n;
    if (y == n / 2) return 0;
    double aky = fabs(c->ky[y]);
    return aky <= (double)c->kymax[a];
}

/* geometry: init.f:15-29, mpisetup.f:307-357 (cut_z, xz_tot), next_xz
 * (mpisetup.f:710-732), masks.f:46-83 */
static void geom_build(orc_ctx *c)
{
    int n = c->n;
    c->kx = (double *)malloc(sizeof(double) * (size_t)(n / 2 + 1));
    c->ky = (double *)malloc(sizeof(double) * (size_t)n);
    c->kz = (double *)malloc(sizeof(double) * (size_t)n);
    for (int x = 0; x <= n / 2; x++) c->kx[x] = x;
    for (int y = 0; y < n; y++) c->ky[y] = (y > n / 2) ? y - n : y;
    for (int z = 0; z < n; z++) c->kz[z] = (z > n / 2) ? z - n : z;

    int ikmax = (int)((double)n * sqrt(2.0) / 3.0);
    int kxn = ikmax + 1;
    if (kxn > n / 2) kxn = n / 2;
    c->kxn = kxn;
    c->cut = (int *)malloc(sizeof(int) * (size_t)kxn);
    c->kc = (int *)malloc(sizeof(int) * (size_t)kxn);
    c->colstart = (int *)malloc(sizeof(int) * (size_t)(kxn + 1));
    double rnxi = 1.0 / n;
    int tot = 0;
    for (int x = 0; x < kxn; x++) {
        double t = c->kx[x] * rnxi;
        double rc = n * (1.0 - 2.0 * sqrt(2.0 / 9.0 - t * t));
        int cc = (int)(rc / 2);
        c->cut[x] = cc;
        c->kc[x] = n / 2 - 1 - cc;
        c->colstart[x] = tot;
        tot += n - 1 - cc * 2;
    }
    c->colstart[kxn] = tot;
    c->xz_tot = tot;
    c->ax = (int *)malloc(sizeof(int) * (size_t)tot);
    c->az = (int *)malloc(sizeof(int) * (size_t)tot);
    c->kymax = (int *)malloc(sizeof(int) * (size_t)tot);
    double two9 = 2. / 9.;
    double rnyi = 1. / n, rnzi = 1. / n;
    for (int x = 0; x < kxn; x++) {
        int kcx = c->kc[x];
        for (int i = 0; i < 2 * kcx + 1; i++) {
            int a = c->colstart[x] + i;
            int kz = (i <= kcx) ? i : i - (2 * kcx + 1);
            int z = (kz < 0) ? kz + n : kz;
            c->ax[a] = x;
            c->az[a] = z;
            double sqkx = (c->kx[x] * rnxi) * (c->kx[x] * rnxi);
            double tz = c->kz[z] * rnzi;
            double sqkz = tz * tz + sqkx;
            int km = -1;
            for (int m = 0; m <= n / 2; m++) {
                double ty = m * rnyi;
                double sqk = ty * ty + sqkz;
                if (sqk > two9) break;
                km = m;
            }
            c->kymax[a] = km;
        }
    }
}

orc_ctx *orc_create(int n, double viscos, double cfl, double dt, int kshift,
                    int seed_input, int ksran, double beta1, double beta2, double beta3)
{
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    c->n = n;
    c->viscos = viscos; c->cfl = cfl; c->dt0 = dt; c->dt = dt;
    c->kshift = kshift; c->ksran = ksran;
    c->b11 = beta1 * beta1; c->b22 = beta2 * beta2; c->b33 = beta3 * beta3;
    c->beta[0] = beta1; c->beta[1] = beta2; c->beta[2] = beta3;
    c->pr = 1.0;
    rng_init(&c->rng, seed_input);
    geom_build(c);
    size_t nst = (size_t)3 * c->xz_tot * n;
    c->u = (cx *)calloc(nst, sizeof(cx));
    c->un = (cx *)calloc(nst, sizeof(cx));
    c->sx = (cx *)calloc((size_t)2 * n, sizeof(cx));
    c->sy = (cx *)calloc((size_t)2 * n, sizeof(cx));
    c->sz = (cx *)calloc((size_t)2 * n, sizeof(cx));
    c->xfac = (double *)calloc((size_t)n, sizeof(double));
    c->yfac = (double *)calloc((size_t)n, sizeof(double));
    c->zfac = (double *)calloc((size_t)n, sizeof(double));
    c->xdif = (double *)calloc((size_t)n, sizeof(double));
    c->ydif = (double *)calloc((size_t)n, sizeof(double));
    c->zdif = (double *)calloc((size_t)n, sizeof(double));
    tw_make(&c->tw, n);
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    free(c->kx); free(c->ky); free(c->kz); free(c->cut); free(c->kc); free(c->colstart);
    free(c->ax); free(c->az); free(c->kymax); free(c->u); free(c->un); free(c->u1);
    free(c->sx); free(c->sy); free(c->sz); free(c->xfac); free(c->yfac); free(c->zfac);
    free(c->xdif); free(c->ydif); free(c->zdif);
    free(c->tw.w);
    free(c->pp);
    free(c->suo); free(c->svo); free(c->velinc); free(c->w1); free(c->w2); free(c->forc); free(c->efkz);
    free(c);
}

int orc_kxn(orc_ctx *c) { return c->kxn; }
int orc_xz_tot(orc_ctx *c) { return c->xz_tot; }
void orc_geometry(orc_ctx *c, int *cut, int *colstart, int *kymax, int *az)
{
    memcpy(cut, c->cut, sizeof(int) * (size_t)c->kxn);
    memcpy(colstart, c->colstart, sizeof(int) * (size_t)(c->kxn + 1));
    memcpy(kymax, c->kymax, sizeof(int) * (size_t)c->xz_tot);
    memcpy(az, c->az, sizeof(int) * (size_t)c->xz_tot);
}

/* One passive scalar (nc = 1) with Schmidt number pr and mean gradient
 * grad (input records of input.f; cb = beta * grad, init.f:42-45).  The
 * state grows to 4 variables; the scalar starts at zero (incond.f:49). */
void orc_set_scalar(orc_ctx *c, int nc, double pr, double g1, double g2, double g3)
{
    size_t vs = (size_t)c->xz_tot * c->n;
    c->nc = nc ? 1 : 0;
    c->pr = pr;
    c->cb[0] = c->beta[0] * g1; c->cb[1] = c->beta[1] * g2; c->cb[2] = c->beta[2] * g3;
    c->u = (cx *)realloc(c->u, sizeof(cx) * (3 + c->nc) * vs);
    c->un = (cx *)realloc(c->un, sizeof(cx) * (3 + c->nc) * vs);
    if (c->nc) {
        memset(c->u + 3 * vs, 0, sizeof(cx) * vs);
        memset(c->un + 3 * vs, 0, sizeof(cx) * vs);
    }
}

/* state I/O: [3+nc][xz_tot][n] complex (re,im interleaved), the reference's
 * uy(ny,num_al,3+nc) layout.  set_state copies un into both un and u
 * (incond.f:146). */
void orc_set_state(orc_ctx *c, const double *un)
{
    size_t nst = (size_t)(3 + c->nc) * c->xz_tot * c->n;
    memcpy(c->un, un, nst * sizeof(cx));
    memcpy(c->u, un, nst * sizeof(cx));
}

void orc_get_state(orc_ctx *c, double *u, double *un)
{
    size_t nst = (size_t)(3 + c->nc) * c->xz_tot * c->n;
    if (u) memcpy(u, c->u, nst * sizeof(cx));
    if (un) memcpy(un, c->un, nst * sizeof(cx));
}

void orc_get_scalars(orc_ctx *c, double *out)
{
    out[0] = c->dt; out[1] = c->time; out[2] = c->velmax; out[3] = c->dt2;
    out[4] = c->gsh[0][0]; out[5] = c->gsh[1][0]; out[6] = c->gsh[2][0];
    out[7] = c->gsh[0][1]; out[8] = c->gsh[1][1]; out[9] = c->gsh[2][1];
    out[10] = (double)c->status;
}

/* ------------------------------------------------------------------------ */
/* shifts.f:40-178 (kshift 1..4) as compiled with -DRKFOUR (the makefile's  */
/* configuration), which also draws gsh(:,3:4) each step.                   */
/* ------------------------------------------------------------------------ */
static double cancel(double d) { return fmod(d + 0.5, 1.); }

static void shifts(orc_ctx *c)
{
    int n = c->n;
    int ks = c->kshift;
    if (c->jstep == 1 && (ks == 1 || ks == 3)) {
        rng_ranseq(&c->rng, c->ksran);
        for (int i = 0; i < 3; i++) c->gsh[i][1] = rng_ranu(&c->rng);
        for (int i = 0; i < 3; i++) c->gsh4[i][1] = rng_ranu(&c->rng);
    }
    if (ks == 1 || ks == 2) rng_ranseq(&c->rng, c->ksran);
    for (int i = 0; i < 3; i++) {
        if (ks == 1) { c->gsh[i][0] = cancel(c->gsh[i][1]); c->gsh[i][1] = rng_ranu(&c->rng); }
        else if (ks == 2) { c->gsh[i][0] = rng_ranu(&c->rng); c->gsh[i][1] = cancel(c->gsh[i][0]); }
        else if (ks == 3) { c->gsh[i][0] = cancel(c->gsh[i][1]); c->gsh[i][1] = cancel(c->gsh[i][0]); }
        else { c->gsh[i][0] = 0.; c->gsh[i][1] = 0.; }
    }
    for (int i = 0; i < 3; i++) {
        if (ks == 1) { c->gsh4[i][0] = cancel(c->gsh4[i][1]); c->gsh4[i][1] = rng_ranu(&c->rng); }
        else if (ks == 2) { c->gsh4[i][0] = rng_ranu(&c->rng); c->gsh4[i][1] = cancel(c->gsh4[i][0]); }
        else if (ks == 3) { c->gsh4[i][0] = cancel(c->gsh4[i][1]); c->gsh4[i][1] = cancel(c->gsh4[i][0]); }
        else { c->gsh4[i][0] = 0.; c->gsh4[i][1] = 0.; }
    }
    double pi = 4. * atan(1.);
    double ph = 2. * pi / n;
    for (int k = 0; k < 2; k++) {
        for (int x = 0; x <= n / 2 && x < n; x++) {
            double th = (ph * c->kx[x]) * c->gsh[0][k];
            c->sx[k * n + x] = cmk(cos(th), sin(th));
        }
        for (int y = 0; y < n; y++) {
            double th = (ph * c->ky[y]) * c->gsh[1][k];
            c->sy[k * n + y] = cmk(cos(th), sin(th));
        }
        for (int z = 0; z < n; z++) {
            double th = (ph * c->kz[z]) * c->gsh[2][k];
            c->sz[k * n + z] = cmk(cos(th), sin(th));
        }
    }
}

/* Externally supplied grid shifts (for tests that drive stages directly). */
void orc_set_shifts(orc_ctx *c, const double *gsh /* [3][2] */)
{
    int n = c->n;
    for (int i = 0; i < 3; i++) { c->gsh[i][0] = gsh[2 * i]; c->gsh[i][1] = gsh[2 * i + 1]; }
    double pi = 4. * atan(1.);
    double ph = 2. * pi / n;
    for (int k = 0; k < 2; k++) {
        for (int x = 0; x <= n / 2 && x < n; x++) {
            double th = (ph * c->kx[x]) * c->gsh[0][k];
            c->sx[k * n + x] = cmk(cos(th), sin(th));
        }
        for (int y = 0; y < n; y++) {
            double th = (ph * c->ky[y]) * c->gsh[1][k];
            c->sy[k * n + y] = cmk(cos(th), sin(th));
        }
        for (int z = 0; z < n; z++) {
            double th = (ph * c->kz[z]) * c->gsh[2][k];
            c->sz[k * n + z] = cmk(cos(th), sin(th));
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Stage pieces                                                             */
/* ------------------------------------------------------------------------ */

/* phshift_inplace (phshift.f:71-135): uy *= sy(y)*(sx(x)*sz(z)); masked -> 0 */
static void phase_shift(orc_ctx *c, cx *u, int nv, int ks)
{
    int n = c->n;
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < c->xz_tot; a++) {
        cx sxz = cmul(c->sx[ks * n + c->ax[a]], c->sz[ks * n + c->az[a]]);
        for (int y = 0; y < n; y++) {
            if (mask_ok(c, a, y)) {
                cx sh = cmul(c->sy[ks * n + y], sxz);
                for (int v = 0; v < nv; v++) {
                    cx *p = &u[((size_t)v * c->xz_tot + a) * n + y];
                    *p = cmul(*p, sh);
                }
            } else {
                for (int v = 0; v < nv; v++) u[((size_t)v * c->xz_tot + a) * n + y] = CZERO;
            }
        }
    }
}

/* itransform_vel.f:11-129 with kxcomm1_clean.f (y backward FFT, scatter to z
 * pencils with zero fill of the cut band, :205-255), the z backward FFT with
 * the Nyquist row zeroed (itransform_vel.f:80-94) and kxcomm2.f (x backward
 * complex-to-real, kx >= kxn zero padded, :308-321).
 * nv = 6 carries one scalar: u[3] = its y gradient, u[4] and u[5] the
 * shifted scalar, multiplied in the z pencils by i b11 kx and i b33 kz
 * (itransform.f:188-198).
 * in: u[v][a][y] (overwritten: y transformed), out: p[v][y][z][x] real. */
static void itransform(orc_ctx *c, cx *u, int nv, double *p)
{
    int n = c->n, kxn = c->kxn, tot = c->xz_tot;
    /* y backward */
    #pragma omp parallel
    {
        cx *tmp = (cx *)malloc(sizeof(cx) * (size_t)n);
        #pragma omp for schedule(static)
        for (long l = 0; l < (long)nv * tot; l++) fft_line(u + l * n, tmp, n, +1, &c->tw);
        free(tmp);
    }
    /* z pencils: zl[v][y][x][z] */
    cx *zl = (cx *)calloc((size_t)nv * n * kxn * n, sizeof(cx));
    #pragma omp parallel
    {
        cx *tmp = (cx *)malloc(sizeof(cx) * (size_t)n);
        #pragma omp for schedule(static) collapse(2)
        for (int v = 0; v < nv; v++)
            for (int y = 0; y < n; y++)
                for (int x = 0; x < kxn; x++) {
                    cx *line = zl + (((size_t)v * n + y) * kxn + x) * n;
                    for (int a = c->colstart[x]; a < c->colstart[x + 1]; a++)
                        line[c->az[a]] = u[((size_t)v * tot + a) * n + y];
                    line[n / 2] = CZERO;
                    if (nv == 6 && v == 4) {
                        cx bk1i = cmk(0.0, c->b11 * c->kx[x]);
                        for (int z = 0; z < n; z++) if (z != n / 2) line[z] = cmul(bk1i, line[z]);
                    } else if (nv == 6 && v == 5) {
                        for (int z = 0; z < n; z++)
                            if (z != n / 2) line[z] = cmul(cmk(0.0, c->b33 * c->kz[z]), line[z]);
                    }
                    fft_line(line, tmp, n, +1, &c->tw);
                }
        free(tmp);
    }
    /* x complex-to-real: Hermitian extension; imaginary part of the kx=0
     * term ignored, as a c2r transform does */
    #pragma omp parallel
    {
        cx *line = (cx *)malloc(sizeof(cx) * (size_t)n);
        cx *tmp = (cx *)malloc(sizeof(cx) * (size_t)n);
        #pragma omp for schedule(static) collapse(2)
        for (int v = 0; v < nv; v++)
            for (int y = 0; y < n; y++)
                for (int z = 0; z < n; z++) {
                    for (int k = 0; k < n; k++) line[k] = CZERO;
                    for (int x = 0; x < kxn; x++) {
                        cx val = zl[(((size_t)v * n + y) * kxn + x) * n + z];
                        if (x == 0) { line[0] = cmk(val.re, 0.0); }
                        else { line[x] = val; line[n - x] = cconj(val); }
                    }
                    fft_line(line, tmp, n, +1, &c->tw);
                    double *out = p + (((size_t)v * n + y) * n + z) * n;
                    for (int x = 0; x < n; x++) out[x] = line[x].re;
                }
        free(line); free(tmp);
    }
    free(zl);
}

/* realspace_vel.f:61-118 (stage 1, with velmax) and :143-178 (stage 2).
 * in: p[0..2] = u,v,w ; out: p[0..4] = b11 u^2 - bv2, uv, b33 w^2 - bv2, vw, uw.
 * With a scalar, in: p[3..5] = its y, x, z gradients; out: p[5] = the
 * advection term u.(cb + grad theta) (itransform.f:522-530). */
static double realspace(orc_ctx *c, double *p, int want_velmax)
{
    int n = c->n;
    size_t np = (size_t)n * n * n;
    double xnorm = c->b11 * n, ynorm = c->b22 * n, znorm = c->b33 * n;
    double vm = 0.;
    #pragma omp parallel for reduction(max:vm) schedule(static)
    for (long i = 0; i < (long)np; i++) {
        double u = p[i], v = p[np + i], w = p[2 * np + i];
        if (c->nc) {
            double gy = p[3 * np + i], gx = p[4 * np + i], gz = p[5 * np + i];
            double term1 = u * (c->cb[0] + gx);
            double term2 = v * (c->cb[1] + gy);
            double term3 = w * (c->cb[2] + gz);
            p[5 * np + i] = term1 + term2 + term3;
        }
        double bv2 = c->b22 * v * v;
        p[4 * np + i] = u * w;
        p[3 * np + i] = v * w;
        if (want_velmax) {
            double vel = xnorm * fabs(u) + ynorm * fabs(v) + znorm * fabs(w);
            if (vel > vm) vm = vel;
        }
        p[2 * np + i] = c->b33 * w * w - bv2;
        p[np + i] = u * v;
        p[i] = c->b11 * u * u - bv2;
    }
    return vm;
}

/* transform.f:10-301: x forward real-to-complex times 1/nx (xkcomm1.f:97,135),
 * z forward FFT (transform.f:129-138), derivative combination
 * (transform.f:230-234, Nyquist z row skipped), cylinder gather keeping
 * |kz| <= kc(x) (xkcomm2.f:96-125) and y forward FFT (xkcomm2.f:229).
 * A scalar's advection term (p[5]) is transformed without derivatives into
 * u[4] (transform.f: i2f = 4 + nc).
 * in: p[5+nc][y][z][x] ; out: u[4+nc][a][y] */
static void transform(orc_ctx *c, const double *p, cx *u)
{
    int n = c->n, kxn = c->kxn, tot = c->xz_tot;
    int nvp = 5 + c->nc;
    double factor = 1. / (double)n;
    cx *zl = (cx *)calloc((size_t)nvp * n * kxn * n, sizeof(cx));
    /* x r2c, scale, transpose to z pencils zl[v][y][x][z] */
    #pragma omp parallel
    {
        cx *line = (cx *)malloc(sizeof(cx) * (size_t)n);
        cx *tmp = (cx *)malloc(sizeof(cx) * (size_t)n);
        #pragma omp for schedule(static) collapse(2)
        for (int v = 0; v < nvp; v++)
            for (int y = 0; y < n; y++)
                for (int z = 0; z < n; z++) {
                    const double *in = p + (((size_t)v * n + y) * n + z) * n;
                    for (int x = 0; x < n; x++) line[x] = cmk(in[x], 0.0);
                    fft_line(line, tmp, n, -1, &c->tw);
                    for (int x = 0; x < kxn; x++)
                        zl[(((size_t)v * n + y) * kxn + x) * n + z] = cscale(factor, line[x]);
                }
        free(line); free(tmp);
    }
    /* z forward */
    #pragma omp parallel
    {
        cx *tmp = (cx *)malloc(sizeof(cx) * (size_t)n);
        #pragma omp for schedule(static)
        for (long l = 0; l < (long)nvp * n * kxn; l++) fft_line(zl + l * n, tmp, n, -1, &c->tw);
        free(tmp);
    }
    /* derivative combination, m = 2 mesh (b11(2) = b11 etc.) */
    size_t vs = (size_t)n * kxn * n;
    #pragma omp parallel for schedule(static) collapse(2)
    for (int y = 0; y < n; y++)
        for (int x = 0; x < kxn; x++) {
            cx bk1i1 = cmk(0.0, c->kx[x]);
            cx bk1i2 = cmk(0.0, c->b11 * c->kx[x]);
            for (int z = 0; z < n; z++) {
                if (z == n / 2) continue;
                cx bk3i1 = cmk(0.0, c->b33 * c->kz[z]);
                cx bk3i2 = cmk(0.0, c->kz[z]);
                size_t o = ((size_t)y * kxn + x) * n + z;
                cx u1 = zl[o], u3 = zl[2 * vs + o], u5 = zl[4 * vs + o];
                zl[o] = cadd(cmul(bk1i1, u1), cmul(bk3i1, u5));
                zl[2 * vs + o] = cadd(cmul(bk1i2, u5), cmul(bk3i2, u3));
            }
        }
    /* cylinder gather (4 variables: slots 1,2,3,4; the scalar term as the
     * fifth, taken from zl variable 5) and y forward */
    #pragma omp parallel
    {
        cx *tmp = (cx *)malloc(sizeof(cx) * (size_t)n);
        #pragma omp for schedule(static) collapse(2)
        for (int v = 0; v < 4 + c->nc; v++)
            for (int a = 0; a < tot; a++) {
                cx *line = u + ((size_t)v * tot + a) * n;
                int x = c->ax[a], z = c->az[a];
                int vz = v < 4 ? v : 5;
                for (int y = 0; y < n; y++) line[y] = zl[(((size_t)vz * n + y) * kxn + x) * n + z];
                fft_line(line, tmp, n, -1, &c->tw);
            }
        free(tmp);
    }
    free(zl);
}

/* step.f:49-99 (dt from CFL), :247-262 (time, dt2), :366-385 (integrating
 * factors; a11=a22=a33=0 so term = b(1)*dt).  Returns nonzero on the abort
 * conditions of step.f:79-84, :280-283, :289-295. */
static int step_control(orc_ctx *c)
{
    int n = c->n;
    c->dt = c->dt0;
    int err = 0;
    if (c->cfl > 0.) {
        c->dt = c->cfl / c->velmax;
        if (c->velmax < .001) err = 1;
    }
    c->time = c->time + c->dt;
    if (c->dt == 0.) err = 2;
    c->dt2 = c->dt / 2.;
    if (c->cfl > 0.) {
        if (c->dt > 10. || c->dt < 1.e-7) err = 3;
    } else if (c->cfl < 0.) {
        double cn = c->velmax * c->dt / 2. / (4. * atan(1.));
        if (cn > 1) err = 4;
    }
    double term = c->b11 * c->dt;
    for (int x = 0; x <= n / 2 && x < n; x++) c->xfac[x] = exp(-(c->viscos * (c->kx[x] * c->kx[x]) * term));
    term = c->b22 * c->dt;
    for (int y = 0; y < n; y++) c->yfac[y] = exp(-(c->viscos * (c->ky[y] * c->ky[y]) * term));
    term = c->b33 * c->dt;
    for (int z = 0; z < n; z++) c->zfac[z] = exp(-(c->viscos * (c->kz[z] * c->kz[z]) * term));
    if (c->nc) {
        /* step.f:387-407 */
        for (int z = 0; z < n; z++) c->zdif[z] = pow(c->zfac[z], 1. / c->pr);
        for (int x = 0; x <= n / 2 && x < n; x++) c->xdif[x] = pow(c->xfac[x], 1. / c->pr);
        for (int y = 0; y < n; y++) c->ydif[y] = pow(c->yfac[y], 1. / c->pr);
    }
    return err;
}

/* wavespace_vel.f:80,163-174: un-shift and finish the y derivatives.
 * in: w[4][a][y]; out: w[0..2] = (dt/2) N(u).  A scalar's term w[4] is
 * un-shifted the same way (wavespace_module.f:344-357); every variable is
 * zero outside the sphere (:289-291). */
static void wavespace(orc_ctx *c, cx *w, int ks)
{
    int n = c->n, tot = c->xz_tot;
    double norm = c->dt2 / n / n;
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];
        cx sxz = cmul(c->sz[ks * n + z], c->sx[ks * n + x]);
        double bk1 = c->b11 * c->kx[x], bk3 = c->b33 * c->kz[z];
        for (int y = 0; y < n; y++) {
            size_t o = (size_t)a * n + y;
            size_t vs = (size_t)tot * n;
            if (mask_ok(c, a, y)) {
                cx s = cconj(cmul(sxz, c->sy[ks * n + y]));
                cx sxyz = cscale(-norm, s);
                cx ib = cmk(0.0, c->b22);
                ib = cscale(c->ky[y], ib);
                cx utmp1 = cmul(ib, sxyz);
                cx u1 = w[o], u2 = w[vs + o], u3 = w[2 * vs + o], u4 = w[3 * vs + o];
                w[o] = cadd(cmul(sxyz, u1), cmul(utmp1, u2));
                cx si = cmul(sxyz, cmk(0.0, 1.0));
                w[vs + o] = cmul(si, cadd(cscale(bk1, u2), cscale(bk3, u4)));
                w[2 * vs + o] = cadd(cmul(sxyz, u3), cmul(utmp1, u4));
                if (c->nc) w[4 * vs + o] = cmul(sxyz, w[4 * vs + o]);
            } else {
                w[o] = CZERO; w[vs + o] = CZERO; w[2 * vs + o] = CZERO; w[3 * vs + o] = CZERO;
                if (c->nc) w[4 * vs + o] = CZERO;
            }
        }
    }
}

static void add_forcing(orc_ctx *c, cx *w, int stage1);

/* pressure projection shared by proc4a.f:553-571 and proc4b.f:85-106 */
static void project(orc_ctx *c, cx *u, int a, int y)
{
    int n = c->n, tot = c->xz_tot;
    int x = c->ax[a], z = c->az[a];
    size_t o = (size_t)a * n + y, vs = (size_t)tot * n;
    double bk1 = c->b11 * c->kx[x];
    double bk3 = c->b33 * c->kz[z];
    double bkk3 = bk3 * c->kz[z];
    double bk12 = bk1 * c->kx[x] + c->b22 * (c->ky[y] * c->ky[y]);
    double den = bk12 + bkk3;
    cx s = cadd(cadd(cscale(bk1, u[o]), cscale(c->b22 * c->ky[y], u[vs + o])), cscale(bk3, u[2 * vs + o]));
    cx psi = cmk(-(s.re / den), -(s.im / den));
    u[o] = cadd(u[o], cscale(c->kx[x], psi));
    u[vs + o] = cadd(u[vs + o], cscale(c->ky[y], psi));
    u[2 * vs + o] = cadd(u[2 * vs + o], cscale(c->kz[z], psi));
}

/* proc4a.f:418-486 (integrating factor, predictor) and :535-573 (projection).
 * The mean mode (k=0) uses factor 1: the reference multiplies it by an
 * unset element of facty, but both terms of that product are zero there. */
static void proc4a(orc_ctx *c, cx *w, cx *un)
{
    int n = c->n, tot = c->xz_tot;
    size_t vs = (size_t)tot * n;
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];
        for (int y = 0; y < n; y++) {
            if (!mask_ok(c, a, y)) continue;
            double f = (a == 0 && y == 0) ? 1.0 : c->xfac[x] * c->yfac[y] * c->zfac[z];
            for (int i = 0; i < 3; i++) {
                size_t o = i * vs + (size_t)a * n + y;
                cx untemp = un[o];
                un[o] = cscale(f, cadd(untemp, w[o]));
                w[o] = cscale(f, cadd(untemp, cscale(2., w[o])));
            }
            if (c->nc) {
                /* proc4a.f:507-522: scalar term in w[4], old scalar in un[3] */
                double fs = c->xdif[x] * c->ydif[y] * c->zdif[z];
                size_t o = (size_t)a * n + y;
                cx untemp = un[3 * vs + o];
                un[3 * vs + o] = cscale(fs, cadd(untemp, w[4 * vs + o]));
                w[4 * vs + o] = cscale(fs, cadd(untemp, cscale(2., w[4 * vs + o])));
            }
            if (a == 0 && y == 0) continue;
            project(c, w, a, y);
        }
    }
    add_forcing(c, w, 1);
}

/* proc4b.f:38-106 (corrector and projection), :183-191 (copy), :200-205
 * (zero mean) */
static void proc4b(orc_ctx *c, cx *w, cx *un)
{
    int n = c->n, tot = c->xz_tot;
    size_t vs = (size_t)tot * n;
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < tot; a++) {
        for (int y = 0; y < n; y++) {
            if (!mask_ok(c, a, y)) continue;
            for (int i = 0; i < 3; i++) {
                size_t o = i * vs + (size_t)a * n + y;
                w[o] = cadd(un[o], w[o]);
            }
            if (c->nc) {
                /* proc4b.f:69-75 */
                size_t o = (size_t)a * n + y;
                w[4 * vs + o] = cadd(un[3 * vs + o], w[4 * vs + o]);
            }
            if (a == 0 && y == 0) continue;
            project(c, w, a, y);
        }
    }
    add_forcing(c, w, 0);
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < tot; a++) {
        for (int y = 0; y < n; y++) {
            if (!mask_ok(c, a, y)) continue;
            for (int i = 0; i < 3; i++) {
                size_t o = i * vs + (size_t)a * n + y;
                un[o] = w[o];
            }
            if (c->nc) un[3 * vs + (size_t)a * n + y] = w[4 * vs + (size_t)a * n + y];
        }
    }
    for (int i = 0; i < 3; i++) { w[i * vs] = CZERO; un[i * vs] = CZERO; }
    if (c->nc) { w[4 * vs] = CZERO; un[3 * vs] = CZERO; }
}


/* RK4 (-DRKFOUR), homogeneous/advanc_1.f..advanc_4.f as written, nc = 0.
 * w holds the stage's wavespace term (dt/2 attached), u1 the accumulator.
 * advanc_1.f:102-117: f = xfac yfac zfac; u1 = f (un + w/3), u = f (un + w);
 *   projection of u (:131-156, the mean mode skipped); forcing with efkz
 *   (:164-216).
 * advanc_2.f/advanc_3.f:46-54: u1 = u1 + w*2/3; u = un + w (stage 2) or
 *   un + w*2 (stage 3); projection of u (:62-82); forcing without the
 *   |k| <= kforce test (:94-141).
 * advanc_4.f:46-54: u1 = u1 + w*1/3; projection of u1 (:62-82); the forcing
 *   is added to u (:94-141) and then overwritten by the copy
 *   un = u = u1 (:149-161); the mean mode of u and un is zeroed (:168-174). */
static void advanc(orc_ctx *c, int kstep, cx *w, cx *un, cx *u1)
{
    int n = c->n, tot = c->xz_tot;
    size_t vs = (size_t)tot * n;
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];
        for (int y = 0; y < n; y++) {
            if (!mask_ok(c, a, y)) continue;
            double f = c->xfac[x] * c->yfac[y] * c->zfac[z];
            for (int i = 0; i < 3; i++) {
                size_t o = i * vs + (size_t)a * n + y;
                cx wv = w[o];
                if (kstep == 1) {
                    cx untemp = un[o];
                    u1[o] = cscale(f, cadd(untemp, cmk(wv.re / 3., wv.im / 3.)));
                    w[o] = cscale(f, cadd(untemp, wv));
                } else if (kstep == 2 || kstep == 3) {
                    u1[o] = cadd(u1[o], cmk(wv.re * 2. / 3., wv.im * 2. / 3.));
                    w[o] = kstep == 2 ? cadd(un[o], wv) : cadd(un[o], cmk(wv.re * 2., wv.im * 2.));
                } else {
                    u1[o] = cadd(u1[o], cmk(wv.re * 1. / 3., wv.im * 1. / 3.));
                }
            }
            if (a == 0 && y == 0) continue;
            project(c, kstep == 4 ? u1 : w, a, y);
        }
    }
    add_forcing(c, w, kstep == 1);
    if (kstep == 4) {
        #pragma omp parallel for schedule(static)
        for (int a = 0; a < tot; a++)
            for (int y = 0; y < n; y++) {
                if (!mask_ok(c, a, y)) continue;
                for (int i = 0; i < 3; i++) {
                    size_t o = i * vs + (size_t)a * n + y;
                    un[o] = u1[o];
                    w[o] = u1[o];
                }
            }
        for (int i = 0; i < 3; i++) { w[i * vs] = CZERO; un[i * vs] = CZERO; }
    }
}

int orc_set_rkmethod(orc_ctx *c, int rk)
{
    if (rk != 2 && rk != 4) return 1;
    if (rk == 4 && c->nc != 0) return 2;
    c->rkmethod = rk;
    if (rk == 4 && !c->u1) c->u1 = (cx *)calloc((size_t)3 * c->xz_tot * c->n, sizeof(cx));
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Eswaran-Pope forcing                                                     */
/* ------------------------------------------------------------------------ */
/* rann2.f:238-254 */
static double erf_as(double x)
{
    double p = .3275911, a1 = .254829592, a2 = -.284496736, a3 = 1.421413741, a4 = -1.453152027, a5 = 1.061405429;
    double t = 1. / (1. + p * fabs(x));
    double q = t * (a1 + t * (a2 + t * (a3 + t * (a4 + t * a5))));
    double e = 1. - q * exp(-x * x);
    if (x < 0.) e = -e;
    return e;
}

/* rann2.f:149-226: inverse-distribution table of the standard normal */
static void rann2_init(orc_ctx *c)
{
    const int ntab = 201, ntabm = 200, ntabmm = 199, ntsq = 201 * 201, ntabh = 100;
    double pi = 3.1415927, rtpii = 0.3989423, rti = 0.7071068;
    double *tab = c->g_tab, *dtab = c->g_dtab;
    double dy = 1. / (double)ntabm;
    double p3 = ntsq * 5.800e-6 - ntab * 4.35160e-3 - 1.7006542;
    double p2 = ntsq * 6.035e-6 - ntab * 4.46257e-3 - 1.8738435;
    double p1 = ntabm * exp(-p2 * p2 / 2.) / sqrt(2. * pi);
    double xmin = 2. * pi * p1 * p1 * 1.e-14;
    xmin = -log(xmin);
    xmin = -sqrt(xmin);
    double xmax = -xmin;
    c->g_p1 = p1;
    tab[1] = xmin; tab[2] = p2; tab[3] = p3;
    tab[ntab] = xmax; tab[ntabm] = -p2; tab[ntabmm] = -p3;
    double y = 2. * dy;
    double xx = tab[3] + dy * (xmax - xmin);
    for (int i = 4; i <= ntabh; i++) {
        y = y + dy;
        double xxmin = tab[i - 1], xxmax = xmax;
        for (int iter = 1; iter <= 50; iter++) {
            double yy = 0.5 * (1. + erf_as(rti * xx));
            double err = yy - y;
            if (fabs(err) < 1.e-6) break;
            if (err > 0.) xxmax = xx;
            if (err < 0.) xxmin = xx;
            double fd = rtpii * exp(-0.5 * xx * xx);
            xx = xx + err / (fd > 1.e-10 ? fd : 1.e-10);
            if (xx <= xxmin || xx >= xxmax) xx = 0.5 * (xxmin + xxmax);
        }
        tab[i] = xx;
    }
    for (int i = 1; i <= ntabh; i++) tab[ntab - i + 1] = -tab[i];
    tab[ntabh + 1] = 0.;
    for (int i = 1; i <= ntabm; i++) dtab[i] = tab[i + 1] - tab[i];
    c->g_ready = 1;
}

/* rann2.f:114-143 with ranu2.f/vrand.f as the uniform source (the ranu LCG) */
static void rann2(orc_ctx *c, double *x, int n)
{
    if (!c->g_ready) rann2_init(c);
    const int ntabm = 200;
    double pi = 3.1415927, azer = 1.e-20, p1 = c->g_p1;
    for (int j = 0; j < n; j++) x[j] = rng_ranu(&c->rng);
    for (int j = 0; j < n; j++) {
        double y = x[j] * ntabm + 1;
        int i = (int)y;
        if (i == 1) {
            double y1 = x[j];
            y1 = 2. * pi * p1 * p1 * y1 * y1;
            if (y1 <= 0.) y1 = azer;
            x[j] = -sqrt(-log(y1));
        } else if (i == ntabm) {
            double y1 = 1. - x[j];
            y1 = 2. * pi * p1 * p1 * y1 * y1;
            x[j] = sqrt(-log(y1));
        } else {
            y = y - i;
            x[j] = c->g_tab[i] + y * c->g_dtab[i];
        }
    }
}

void orc_set_forcing(orc_ctx *c, double kforce, double tforce, double epsfor, double tfiuo, int kranf1, int kranf2)
{
    c->kforce = kforce; c->tforce = tforce; c->epsfor = epsfor; c->tfiuo = tfiuo;
    c->kranf1 = kranf1; c->kranf2 = kranf2;
    double bmin = sqrt(c->b11) < sqrt(c->b22) + sqrt(c->b33) ? sqrt(c->b11) : sqrt(c->b22) + sqrt(c->b33);
    c->kfor = (int)(kforce / bmin + 1.5);                 /* param_set.f:33 */
    c->k2fo = 2 * c->kfor - 1;
    c->nrproc = 4 * c->kfor * c->k2fo * c->k2fo;          /* param_set.f:87 */
    c->ffirst = 1;
    c->suo = (double *)calloc((size_t)c->nrproc, sizeof(double));
    c->svo = (double *)calloc((size_t)c->nrproc, sizeof(double));
    c->velinc = (double *)calloc((size_t)c->nrproc, sizeof(double));
    c->w1 = (double *)calloc((size_t)c->nrproc, sizeof(double));
    c->w2 = (double *)calloc((size_t)c->nrproc, sizeof(double));
    c->forc = (cx *)calloc((size_t)c->kfor * c->k2fo * c->k2fo * 3, sizeof(cx));
    c->efkz = (double *)calloc((size_t)3 * (c->kfor + 2), sizeof(double));
}

/* raniuo.f:56-109 */
static void raniuo(orc_ctx *c, double dtv)
{
    int n = c->nrproc;
    if (c->t1 <= 0. || c->t2 <= 0.) return;
    double diff = fabs(c->t1 / c->t2 - 1.);
    if (diff < 0.05) c->t1 = 0.95 * c->t2;
    if (dtv < 0.) {
        double rr = c->t1 / (c->t1 + c->t2), be = sqrt(rr), ga = sqrt(1. - rr);
        rann2(c, c->w1, n);
        rann2(c, c->w2, n);
        for (int i = 0; i < n; i++) { c->suo[i] = c->w1[i]; c->svo[i] = be * c->w1[i] + ga * c->w2[i]; }
        return;
    }
    double om1 = 1. / c->t1, om2 = 1. / c->t2, s = om1 + om2, d = om2 - om1;
    double a = exp(-om1 * dtv), b = exp(-om2 * dtv), cc = (a - b) / d;
    double sco = cc * sqrt(s * om2), r = sqrt(om2 / s);
    double uu = 1. - a * a;
    double vv = 1. - b * b + 4. * om1 * om2 * b * cc / d - om2 * s * (a * a - b * b) / (d * d);
    double uv = r * (1. - a * b - s * a * cc);
    double al = sqrt(uu), be = uv / al;
    double g2 = vv - be * be;
    double ga = sqrt(g2 > 0. ? g2 : 0.);
    rann2(c, c->w1, n);
    rann2(c, c->w2, n);
    for (int i = 0; i < n; i++) {
        c->svo[i] = b * c->svo[i] + sco * c->suo[i] + be * c->w1[i] + ga * c->w2[i];
        c->suo[i] = a * c->suo[i] + al * c->w1[i];
    }
}

/* force.f:60-166 with vfuo.f:25-55 / vfiuo.f:33-57 */
static void force(orc_ctx *c)
{
    if (c->kforce == 0.) return;
    int n = c->nrproc, kfor = c->kfor, k2fo = c->k2fo, nn = c->n;
    double dt = c->dt;
    if (c->tforce * c->tfiuo == 0.) {
        if (c->ffirst) {
            c->ffirst = 0;
            rng_ranseq(&c->rng, c->kranf1);
            rann2(c, c->suo, n);
        }
        double exp1 = 0.;
        if (c->tforce > 0.05 * dt) exp1 = exp(-dt / c->tforce);
        double exp2 = exp1 * exp1;
        double rana = sqrt(1. - exp2);
        double ranua = sqrt(c->epsfor * c->tforce) * ((1. - exp1) * (1. - exp1)) / sqrt(1. - exp2);
        double ranub = (c->epsfor * (2. * dt + c->tforce * (-3. + 4. * exp1 - exp2)) - ranua * ranua);
        ranub = sqrt(ranub > 0. ? ranub : 0.);
        double ranud = sqrt(c->epsfor * c->tforce) * (1. - exp1);
        rng_ranseq(&c->rng, c->kranf2);
        rann2(c, c->w1, n);
        rann2(c, c->w2, n);
        for (int i = 0; i < n; i++) {
            c->velinc[i] = ranud * c->suo[i] + ranua * c->w1[i] + ranub * c->w2[i];
            c->suo[i] = exp1 * c->suo[i] + rana * c->w1[i];
        }
    } else {
        if (c->ffirst) {
            c->ffirst = 0;
            double q = sqrt(1. - 4. * fabs(c->tfiuo) * fabs(c->tfiuo));
            c->t1 = 0.5 * c->tforce * (1. + q);
            c->t2 = 0.5 * c->tforce * (1. - q);
            c->siga = sqrt(c->epsfor / c->tforce);
            if (c->tfiuo > 0.) { rng_ranseq(&c->rng, c->kranf1); raniuo(c, -1.); }
        }
        rng_ranseq(&c->rng, c->kranf2);
        raniuo(c, dt);
        double fmult = c->siga * dt;
        for (int i = 0; i < n; i++) c->velinc[i] = c->svo[i] * fmult;
    }
    double s1 = sqrt(c->b11), s2 = sqrt(c->b22), s3 = sqrt(c->b33);
#define FOR(x, y, z, i) c->forc[((((size_t)(i) - 1) * k2fo + ((z) - 1)) * k2fo + ((y) - 1)) * kfor + ((x) - 1)]
    for (int z = 1; z <= k2fo; z++)
        for (int y = 1; y <= k2fo; y++) {
            int iy = y + (y / (kfor + 1)) * (nn - k2fo), iz = z + (z / (kfor + 1)) * (nn - k2fo);
            double k2u = s2 * c->ky[iy - 1], k3u = s3 * c->kz[iz - 1];
            for (int x = 1; x <= kfor; x++) {
                size_t o = 2 * ((size_t)(x - 1) + (size_t)kfor * ((y - 1) + (size_t)k2fo * (z - 1)));
                cx alpha = cmk(c->velinc[2 * o], c->velinc[2 * o + 1]);
                cx beta = cmk(c->velinc[2 * o + 2], c->velinc[2 * o + 3]);
                double k1u = s1 * c->kx[x - 1];
                double k = sqrt(k1u * k1u + k2u * k2u + k3u * k3u);
                double k12 = sqrt(k1u * k1u + k2u * k2u);
                if (k > c->kforce || k == 0.) {
                    FOR(x, y, z, 1) = CZERO; FOR(x, y, z, 2) = CZERO; FOR(x, y, z, 3) = CZERO;
                } else if (k12 == 0.) {
                    FOR(x, y, z, 1) = cmk(alpha.re / s1, alpha.im / s1);
                    FOR(x, y, z, 2) = cmk(beta.re / s2, beta.im / s2);
                    FOR(x, y, z, 3) = CZERO;
                } else {
                    double d1 = k * k12 * s1, d2 = k * k12 * s2, d3 = k * s3;
                    cx t1 = cadd(cscale(k2u, cscale(k, alpha)), cscale(k3u, cscale(k1u, beta)));
                    cx t2 = csub(cscale(k3u, cscale(k2u, beta)), cscale(k1u, cscale(k, alpha)));
                    cx t3 = cscale(k12, beta);
                    FOR(x, y, z, 1) = cmk(t1.re / d1, t1.im / d1);
                    FOR(x, y, z, 2) = cmk(t2.re / d2, t2.im / d2);
                    FOR(x, y, z, 3) = cmk(-(t3.re / d3), -(t3.im / d3));
                }
            }
        }
    for (int i = 1; i <= 3; i++) {
        for (int y = kfor + 1; y <= k2fo; y++) FOR(1, y, 1, i) = cconj(FOR(1, k2fo + 2 - y, 1, i));
        for (int z = kfor + 1; z <= k2fo; z++) {
            FOR(1, 1, z, i) = cconj(FOR(1, 1, k2fo + 2 - z, i));
            for (int y = 2; y <= k2fo; y++) FOR(1, y, z, i) = cconj(FOR(1, k2fo + 2 - y, k2fo + 2 - z, i));
        }
    }
#undef FOR
}

/* the forcing addition of proc4a.f:588-651 (stage 1, with efkz and the
 * |k| <= kforce test) and proc4b.f:118-163 (stage 2) */
static void add_forcing(orc_ctx *c, cx *w, int stage1)
{
    if (c->kforce == 0.) return;
    int n = c->n, tot = c->xz_tot, kfor = c->kfor, k2fo = c->k2fo;
    size_t vs = (size_t)tot * n;
    if (stage1) memset(c->efkz, 0, sizeof(double) * 3 * (kfor + 2));
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];   /* 0-based */
        int zz = z + 1, iz;
        if (zz <= kfor) iz = zz; else if (zz >= n + 2 - kfor) iz = zz - n + k2fo; else iz = 0;
        if (iz == 0 || x + 1 > kfor) continue;
        for (int i = 0; i < 3; i++)
            for (int y = 0; y < n; y++) {
                if (!mask_ok(c, a, y)) continue;
                int yy = y + 1, iy;
                if (yy <= kfor) iy = yy; else if (yy >= n + 2 - kfor) iy = yy - n + k2fo; else iy = 0;
                if (iy == 0) continue;
                cx f = c->forc[(((size_t)i * k2fo + (iz - 1)) * k2fo + (iy - 1)) * kfor + x];
                size_t o = i * vs + (size_t)a * n + y;
                if (stage1) {
                    double rks = c->kx[x] * c->kx[x] * c->b11 + c->ky[y] * c->ky[y] * c->b22 + c->kz[z] * c->kz[z] * c->b33;
                    if (!(rks <= c->kforce * c->kforce)) continue;
                    int k = (int)(sqrt(rks) + 1.5);
                    double term = w[o].re * f.re + w[o].im * f.im;
                    double tfact = (x == 0) ? 1. : 2.;
                    double ssq = i == 0 ? c->b11 : (i == 1 ? c->b22 : c->b33);
                    c->efkz[(k - 1) * 3 + i] += 2. * term * tfact * ssq;
                }
                w[o] = cadd(w[o], f);
            }
    }
}

void orc_get_forcing(orc_ctx *c, double *table, double *efkz)
{
    if (table) memcpy(table, c->forc, sizeof(cx) * (size_t)c->kfor * c->k2fo * c->k2fo * 3);
    if (efkz) memcpy(efkz, c->efkz, sizeof(double) * 3 * (size_t)c->kfor);
}

/* Gaussian numbers of rann2 from the given LCG sequence (tests) */
void orc_rann2(orc_ctx *c, int seq, double *x, int n)
{
    rng_ranseq(&c->rng, seq);
    rann2(c, x, n);
}


/* ------------------------------------------------------------------------ */
/* Lagrangian particles (LAG_LOCAL)                                         */
/* ------------------------------------------------------------------------ */
/* solsp1.f:21-40: factors of the periodic [1 4 1] system */
static void solsp1(int n, double *p, double *q, double *t, double *d)
{
    double *s = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    q[0] = 0.;
    for (int i = 1; i <= n; i++) { p[i] = q[i - 1] + 4.; q[i] = -1. / p[i]; }
    s[0] = 1.;
    for (int i = 1; i <= n; i++) s[i] = -s[i - 1] / p[i];
    t[n] = 1.;
    for (int i = n - 1; i >= 1; i--) t[i] = q[i] * t[i + 1] + s[i];
    *d = 1. / (t[1] + t[n - 1] + 4.);
    for (int i = 1; i <= n; i++) p[i] = 1. / p[i];
    free(s);
}

/* splx.f:20-40 on one line: f[1..n] (1-based) -> b[1..n+3]; scale multiplies
 * the input (splz_m.f:31 uses 216) */
static void spl_line(int n, const double *p, const double *q, const double *t, double d, const double *f,
                     double scale, double *u, double *v, double *b)
{
    u[0] = 0.; v[n] = 0.;
    for (int x = 1; x <= n; x++) u[x] = (f[x] * scale - u[x - 1]) * p[x];
    for (int x = n - 1; x >= 1; x--) v[x] = q[x] * v[x + 1] + u[x];
    b[n + 1] = d * (f[n] * scale - v[1] - v[n - 1]);
    for (int x = n - 1; x >= 1; x--) b[x + 1] = t[x] * b[n + 1] + v[x];
    b[1] = b[n + 1]; b[n + 2] = b[2]; b[n + 3] = b[3];
}

/* spxyz_m.f: x sweep, z sweep (x216), y sweep of one variable.
 * in: f[y][z][x] (0-based, n^3); out: bs[y+1][z+1][x+1] over (n+3)^3, index
 * j in 1..n+3 holding grid point j-2 (mod n) */
static void spline3(orc_ctx *c, const double *f, double *bs)
{
    int n = c->n, nb = n + 3;
    double *p = malloc(sizeof(double) * (n + 1)), *q = malloc(sizeof(double) * (n + 1)), *t = malloc(sizeof(double) * (n + 1));
    double d;
    solsp1(n, p, q, t, &d);
    double *A = calloc((size_t)nb * nb * nb, sizeof(double));   /* after x: [y][z][xb] */
    #pragma omp parallel
    {
        double *fl = malloc(sizeof(double) * (n + 4)), *u = malloc(sizeof(double) * (n + 4)),
               *v = malloc(sizeof(double) * (n + 4)), *b = malloc(sizeof(double) * (n + 4));
        #pragma omp for collapse(2)
        for (int y = 0; y < n; y++)
            for (int z = 0; z < n; z++) {
                for (int x = 0; x < n; x++) fl[x + 1] = f[((size_t)y * n + z) * n + x];
                spl_line(n, p, q, t, d, fl, 1.0, u, v, b);
                for (int xb = 1; xb <= nb; xb++) A[(((size_t)(y + 1)) * nb + (z + 1)) * nb + xb - 1] = b[xb];
            }
        /* z sweep (x216) for every x index of the padded x dimension */
        #pragma omp for collapse(2)
        for (int y = 0; y < n; y++)
            for (int xb = 0; xb < nb; xb++) {
                for (int z = 0; z < n; z++) fl[z + 1] = A[(((size_t)(y + 1)) * nb + (z + 1)) * nb + xb];
                spl_line(n, p, q, t, d, fl, 216., u, v, b);
                for (int zb = 1; zb <= nb; zb++) A[(((size_t)(y + 1)) * nb + (zb - 1)) * nb + xb] = b[zb];
            }
        /* y sweep */
        #pragma omp for collapse(2)
        for (int zb = 0; zb < nb; zb++)
            for (int xb = 0; xb < nb; xb++) {
                for (int y = 0; y < n; y++) fl[y + 1] = A[(((size_t)(y + 1)) * nb + zb) * nb + xb];
                spl_line(n, p, q, t, d, fl, 1.0, u, v, b);
                for (int yb = 1; yb <= nb; yb++) bs[(((size_t)(yb - 1)) * nb + zb) * nb + xb] = b[yb];
            }
        free(fl); free(u); free(v); free(b);
    }
    free(A); free(p); free(q); free(t);
}

/* spcal_local.f:175-231: cell index and basis functions along one axis */
static void bweights(double pos, double gfn, int n, int *ib, double w[4])
{
    double px1 = pos - gfn;
    double px = px1 - (double)n;
    long ipx = (long)floor(px);
    long jpx = ipx;
    if (ipx < 0) jpx = ipx + 1000L * n;
    long jloc = jpx % n;
    double bfp = (double)jloc + px - (double)ipx;
    *ib = (int)bfp;
    double t = bfp - *ib, d6 = 1. / 6., tt = 2. / 3.;
    double ym = 1. - t, yms = ym * ym;
    w[0] = ym * yms * d6;
    w[1] = tt + 0.5 * t * (yms - 1.);
    w[3] = t * t * t * d6;
    w[2] = 1. - w[0] - w[1] - w[3];
}

/* spcal_local.f:234-367: sum of the 4x4x4 stencil; bs index kk = ib+k,
 * folded by nb (n+3) */
static double binterp(const double *bs, int n, const double p[3], const double gfn[3])
{
    int nb = n + 3, ib[3];
    double w[3][4];
    for (int j = 0; j < 3; j++) bweights(p[j], gfn[j], n, &ib[j], w[j]);
    double sum = 0.;
    for (int k = 1; k <= 4; k++) {
        int kz = ib[2] + k; if (kz > nb) kz -= nb;
        for (int jj = 1; jj <= 4; jj++) {
            int ky = ib[1] + jj; if (ky > nb) ky -= nb;
            for (int i = 1; i <= 4; i++) {
                int kx = ib[0] + i; if (kx > nb) kx -= nb;
                sum += bs[(((size_t)(ky - 1)) * nb + (kz - 1)) * nb + (kx - 1)] * w[0][i - 1] * w[1][jj - 1] * w[2][k - 1];
            }
        }
    }
    return sum;
}

/* hooks/LAG_LOCAL/partin.f:93-131 (pstart = 0: uniform random positions,
 * nearly equal numbers per y-slice, from the kipran sequence through ranu2,
 * ranu2.f with RANDOM_SEED sharing the seed of ranu) and :141-190 (pstart =
 * -1: a cubic lattice of nop^3 grid nodes); grid planes gx(i) = 1 + (i-1)/
 * beta1 + gsh(1,1) (partsp.f:44-53), box lengths nx, ny, nz (partsp.f:61).
 * Made when the first particle phase runs (partsp.f:147-149), with that
 * step's stage-1 shifts. */
static void partin(orc_ctx *c)
{
    int n = c->n;
    double ps1 = sqrt(c->b11), ps2 = sqrt(c->b22), ps3 = sqrt(c->b33);
    double gx1 = 1. + 0. / ps1 + c->gsh[0][0];
    double gz1 = 1. + 0. / ps3 + c->gsh[2][0];
    long nop = c->pin_nop;
    if (c->pin_pstart == -1) nop = nop * nop * nop;
    free(c->pp);
    c->pp = calloc((size_t)9 * nop, sizeof(double));
    c->np = nop;
    double *pp = c->pp;
    if (c->pin_pstart == 0) {
        long npy = nop / n, npe = nop - npy * n, niny = 0;
        rng_ranseq(&c->rng, c->pin_kipran);
        for (int y = 1; y <= n; y++) {
            long ni = npy + (y <= npe ? 1 : 0);
            for (int k = 0; k < 3; k++)
                for (long i = 0; i < ni; i++) pp[k * nop + niny + i] = rng_ranu(&c->rng);
            double gy = 1. + (double)(y - 1) / ps2 + c->gsh[1][0];
            for (long i = 0; i < ni; i++) {
                long m = niny + i;
                pp[m] = pp[m] * (double)n + gx1;
                pp[nop + m] = pp[nop + m] / ps2 + gy;
                pp[2 * nop + m] = pp[2 * nop + m] * (double)n + gz1;
            }
            niny += ni;
        }
    } else {
        long npu = c->pin_nop;
        long it[3], i1[3], i2[3];
        for (int d = 0; d < 3; d++) {
            it[d] = n / npu + (n % npu ? 1 : 0);
            i1[d] = n / 2 + 1 - npu / 2 * it[d] + it[d] / 2;
            i2[d] = n / 2 + 1 + npu / 2 * it[d] - it[d] / 2;
            if (i1[d] < 1) i1[d] = 1;
            if (i2[d] > n) i2[d] = n;
        }
        double psv[3] = {ps1, ps2, ps3};
        long idx = 0;
        for (long k = i1[2]; k <= i2[2]; k += it[2])
            for (long j = i1[1]; j <= i2[1]; j += it[1])
                for (long i = i1[0]; i <= i2[0]; i += it[0]) {
                    if (idx < nop) {
                        pp[idx] = 1. + (double)(i - 1) / psv[0] + c->gsh[0][0];
                        pp[nop + idx] = 1. + (double)(j - 1) / psv[1] + c->gsh[1][0];
                        pp[2 * nop + idx] = 1. + (double)(k - 1) / psv[2] + c->gsh[2][0];
                    }
                    idx++;
                }
        if (idx != nop) c->status = 5;   /* partin.f:129-135 stops here */
    }
    c->part_first = 1;
    c->pin_nop = 0;
}

void orc_particles_init(orc_ctx *c, long nop, int pstart, int kipran)
{
    c->pin_nop = nop;
    c->pin_pstart = pstart;
    c->pin_kipran = kipran;
}

void orc_particles_set(orc_ctx *c, long np, const double *pos)
{
    free(c->pp);
    c->np = np;
    c->pp = calloc((size_t)9 * np, sizeof(double));
    memcpy(c->pp, pos, sizeof(double) * 3 * (size_t)np);
    c->part_first = 1;
}

void orc_particles_get(orc_ctx *c, double *pos, double *vel)
{
    if (pos) memcpy(pos, c->pp, sizeof(double) * 3 * (size_t)c->np);
    if (vel) memcpy(vel, c->pp + 3 * (size_t)c->np, sizeof(double) * 3 * (size_t)c->np);
}

/* partsp.f:231-299,405-412 with rk_advpos.f and rk_part.f: p[0..2] is the
 * stage-1 physical velocity on the predictor grid; dt is the previous step's */
static void particles_stage1(orc_ctx *c, const double *p)
{
    int n = c->n, nb = n + 3;
    long np = c->np;
    size_t n3 = (size_t)n * n * n, nb3 = (size_t)nb * nb * nb;
    double *bs = malloc(sizeof(double) * 3 * nb3);
    for (int v = 0; v < 3; v++) spline3(c, p + v * n3, bs + v * nb3);
    double gfn[3] = {c->gsh[0][0] + 1., c->gsh[1][0] + 1., c->gsh[2][0] + 1.};
    double pi = 4. * atan(1.);
    double *pp = c->pp;
    if (c->part_first) {
        #pragma omp parallel for
        for (long m = 0; m < np; m++) {
            double x[3] = {pp[m], pp[np + m], pp[2 * np + m]};
            for (int v = 0; v < 3; v++) pp[(3 + v) * np + m] = binterp(bs + v * nb3, n, x, gfn);
        }
        c->part_first = 0;
    } else {
        double fact1 = 0.5 * c->dt / 2. / pi * n * 1.0;
        double fact2 = fact1;
        #pragma omp parallel for
        for (long m = 0; m < np; m++) {
            double x[3], h[3], xs[3], vs[3];
            for (int k = 0; k < 3; k++) {
                h[k] = pp[k * np + m] + fact1 * pp[(3 + k) * np + m];     /* pp(,7:9) */
                xs[k] = h[k] + fact2 * pp[(3 + k) * np + m];
            }
            for (int v = 0; v < 3; v++) vs[v] = binterp(bs + v * nb3, n, xs, gfn);
            for (int k = 0; k < 3; k++) x[k] = h[k] + fact2 * vs[k];
            for (int k = 0; k < 3; k++) pp[k * np + m] = x[k];
            for (int v = 0; v < 3; v++) pp[(3 + v) * np + m] = binterp(bs + v * nb3, n, x, gfn);
        }
    }
    free(bs);
}

/* One RK stage (timestep_module.f:70-481, CLEAN velocity path, nc = 0 or 1).
 * The work array holds u (3 vars; with a scalar also its y gradient and two
 * copies of it, wavespace_module.f:81-97) on entry and the nonlinear slots
 * (4 vars, then the scalar term) after the forward transform; u keeps the
 * result. */
static int rk_stage(orc_ctx *c, int kstep)
{
    int n = c->n, tot = c->xz_tot;
    /* RK4: stages 3 and 4 reuse the shifts of stages 1 and 2
     * (shifts.f:133-136, gsh(:,3) = gsh(:,1), gsh(:,4) = gsh(:,2)) */
    int ks = (kstep - 1) % 2;
    size_t vs = (size_t)tot * n;
    size_t np = (size_t)n * n * n;
    int nc = c->nc;
    phase_shift(c, c->u, 3 + nc, ks);
    cx *w = (cx *)malloc(sizeof(cx) * (4 + 2 * nc) * vs);
    memcpy(w, c->u, sizeof(cx) * 3 * vs);
    if (nc) {
        #pragma omp parallel for schedule(static)
        for (int a = 0; a < tot; a++)
            for (int y = 0; y < n; y++) {
                size_t o = (size_t)a * n + y;
                cx th = c->u[3 * vs + o];
                w[3 * vs + o] = cmul(cmk(0.0, c->b22 * c->ky[y]), th);
                w[4 * vs + o] = th;
                w[5 * vs + o] = th;
            }
    }
    double *p = (double *)malloc(sizeof(double) * (5 + nc) * np);
    itransform(c, w, 3 + 3 * nc, p);
    if (kstep == 1 && c->pin_nop > 0) partin(c);
    if (kstep == 1 && c->np > 0) particles_stage1(c, p);   /* realspace -> lagpart */
    double vm = realspace(c, p, kstep == 1);
    if (kstep == 1) c->velmax = vm;
    transform(c, p, w);
    free(p);
    int err = 0;
    if (kstep == 1) { err = step_control(c); force(c); }
    wavespace(c, w, ks);
    if (c->rkmethod == 4) advanc(c, kstep, w, c->un, c->u1);
    else if (kstep == 1) proc4a(c, w, c->un);
    else proc4b(c, w, c->un);
    memcpy(c->u, w, sizeof(cx) * 3 * vs);
    if (nc) memcpy(c->u + 3 * vs, w + 4 * vs, sizeof(cx) * vs);
    free(w);
    return err;
}

/* One full RK2 step (main.f:392-463: shifts, then timestep).  Returns the
 * step_control status (0 = ok). */
int orc_step(orc_ctx *c)
{
    c->jstep += 1;
    shifts(c);
    int e = rk_stage(c, 1);
    for (int k = 2; k <= (c->rkmethod == 4 ? 4 : 2); k++) {
        int ek = rk_stage(c, k);
        if (!e) e = ek;
    }
    c->status = e;
    return c->status;
}

/* Stage driven with caller-provided shifts (for piecewise tests). */
int orc_stage(orc_ctx *c, int kstep)
{
    return rk_stage(c, kstep);
}

/* sptr.f:119-218 (one-dimensional spectra xrij, yrij, zrij and der2ij of
 * the velocity pairs 11,12,13,22,23,33), :311-346 (normalisation) and
 * :351-468 (correlations, integral scales, rms, Reynolds numbers, eddy
 * turnover times, derivative variances tmij, grdiss, Taylor microscales).
 * xr, yr, zr: [6][n/2+1]; stats[55] in the order corr[6], lijk[6][3],
 * rms[3], raak[3], ett[3], tmij[3][3], grdiss, taak[3][3], tmre[3]. */
void orc_spectra_scales(orc_ctx *c, int which, double *xr, double *yr, double *zr, double *stats)
{
    int n = c->n, tot = c->xz_tot, nh = n / 2 + 1;
    size_t vs = (size_t)tot * n;
    const cx *u = which == 0 ? c->u : c->un;
    int pi_[6] = {0, 0, 0, 1, 1, 2}, pj_[6] = {0, 1, 2, 1, 2, 2};
    double der2[6] = {0, 0, 0, 0, 0, 0};
    memset(xr, 0, sizeof(double) * 6 * nh);
    memset(yr, 0, sizeof(double) * 6 * nh);
    memset(zr, 0, sizeof(double) * 6 * nh);
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];
        double tf = x == 0 ? 1. : 2.;
        for (int ij = 0; ij < 6; ij++) {
            double ysum = 0.;
            for (int y = 0; y < n; y++) {
                if (!mask_ok(c, a, y)) continue;
                cx vi = u[pi_[ij] * vs + (size_t)a * n + y], vj = u[pj_[ij] * vs + (size_t)a * n + y];
                double uiuj = vi.re * vj.re + vi.im * vj.im;
                ysum += uiuj;
                if (y == 0) yr[ij * nh] += uiuj + (tf - 1.) * uiuj;
                else if (y < n / 2) yr[ij * nh + y] += uiuj;
                else yr[ij * nh + (n - y)] += (tf - 1.) * uiuj;
                double ky2 = (y == n / 2) ? 0. : c->b22 * c->ky[y] * c->ky[y];
                der2[ij] += ky2 * (tf * uiuj);
            }
            if (z == 0) zr[ij * nh] += ysum + (tf - 1.) * ysum;
            else if (z < n / 2) zr[ij * nh + z] += ysum;
            else if (z > n / 2) zr[ij * nh + (n - z)] += (tf - 1.) * ysum;
            xr[ij * nh + x] += ysum;
        }
    }
    double sv[3] = {sqrt(c->b11), sqrt(c->b22), sqrt(c->b33)};
    double s23 = sv[1] * sv[2], s31 = sv[2] * sv[0], s12 = sv[0] * sv[1], size = sv[0] * sv[1] * sv[2];
    double pi = 4. * atan(1.), nu = c->viscos, corr[6];
    for (int ij = 0; ij < 6; ij++) {
        double factor = sv[pi_[ij]] * sv[pj_[ij]];
        der2[ij] = der2[ij] * factor;
        for (int k = 0; k < nh; k++) {
            xr[ij * nh + k] = factor * xr[ij * nh + k] / size;
            yr[ij * nh + k] = factor * yr[ij * nh + k] / size;
            zr[ij * nh + k] = factor * zr[ij * nh + k] / size;
        }
    }
    for (int ij = 0; ij < 6; ij++) {
        for (int k = 0; k < nh; k++) {
            xr[ij * nh + k] = s23 * xr[ij * nh + k];
            yr[ij * nh + k] = s31 * yr[ij * nh + k];
            zr[ij * nh + k] = s12 * zr[ij * nh + k];
        }
        double ssum = xr[ij * nh];
        for (int x = 1; x < n / 2; x++) ssum = ssum + 2. * xr[ij * nh + x];
        corr[ij] = sv[0] * ssum;
    }
    double lijk[6][3];
    memset(lijk, 0, sizeof lijk);
    for (int ij = 0; ij < 6; ij++)
        if (corr[ij] != 0.) {
            lijk[ij][0] = pi * xr[ij * nh] / corr[ij];
            lijk[ij][1] = pi * yr[ij * nh] / corr[ij];
            lijk[ij][2] = pi * zr[ij * nh] / corr[ij];
        }
    int kt[3] = {0, 3, 5};
    double rms[3], raak[3] = {0, 0, 0}, ett[3] = {0, 0, 0}, tmij[3][3], taak[3][3], tmre[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++) rms[i] = sqrt(corr[kt[i]]);
    for (int i = 0; i < 3; i++) {
        if (nu > 0.) raak[i] = lijk[kt[i]][i] * rms[i] / nu;
        if (rms[i] != 0.) ett[i] = lijk[kt[i]][i] / rms[i];
        double ssum = 0.;
        for (int x = 1; x < n / 2; x++) ssum = ssum + c->kx[x] * c->kx[x] * xr[kt[i] * nh + x];
        tmij[i][0] = 2. * sv[0] * sv[0] * sv[0] * ssum;
        tmij[i][1] = der2[kt[i]];
        ssum = 0.;
        for (int z = 1; z < n / 2; z++) ssum = ssum + c->kz[z] * c->kz[z] * zr[kt[i] * nh + z];
        tmij[i][2] = 2. * sv[2] * sv[2] * sv[2] * ssum;
    }
    double grdiss = tmij[0][0] + tmij[1][1] + tmij[2][2] + tmij[0][1] + tmij[1][0] + tmij[0][2] + tmij[2][0] +
                    tmij[1][2] + tmij[2][1];
    grdiss = grdiss * nu;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) taak[i][j] = tmij[j][j] != 0. ? sqrt(corr[kt[i]] / tmij[j][j]) : 0.;
    for (int i = 0; i < 3; i++)
        if (nu > 0.) tmre[i] = taak[i][i] * rms[i] / nu;
    double *o = stats;
    for (int ij = 0; ij < 6; ij++) *o++ = corr[ij];
    for (int ij = 0; ij < 6; ij++) for (int a = 0; a < 3; a++) *o++ = lijk[ij][a];
    for (int i = 0; i < 3; i++) *o++ = rms[i];
    for (int i = 0; i < 3; i++) *o++ = raak[i];
    for (int i = 0; i < 3; i++) *o++ = ett[i];
    for (int i = 0; i < 3; i++) for (int a = 0; a < 3; a++) *o++ = tmij[i][a];
    *o++ = grdiss;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) *o++ = taak[i][j];
    for (int i = 0; i < 3; i++) *o++ = tmre[i];
}

/* trfsp.f:62-83,163-170: transfer spectrum of the convective term of u
 * evaluated as at stage 1 on the grid shifted by gsh[3] (itransform,
 * realspace, transform, wavespace with dt/2 = 1, i.e. fmult folded in), dotted
 * with conj(un); tk[k-1], k = 1..n/2. */
void orc_transfer_spectrum(orc_ctx *c, const double *gsh, double *tk)
{
    int n = c->n, tot = c->xz_tot;
    size_t vs = (size_t)tot * n, np = (size_t)n * n * n;
    double save[3][2];
    memcpy(save, c->gsh, sizeof save);
    double g6[6] = {gsh[0], 0., gsh[1], 0., gsh[2], 0.};
    orc_set_shifts(c, g6);
    double dt2 = c->dt2;
    c->dt2 = 1.0;
    cx *w = (cx *)calloc(4 * vs, sizeof(cx));
    memcpy(w, c->u, sizeof(cx) * 3 * vs);
    phase_shift(c, w, 3, 0);
    double *p = (double *)malloc(sizeof(double) * 5 * np);
    itransform(c, w, 3, p);
    int nc = c->nc;
    c->nc = 0;                 /* the velocity path only */
    realspace(c, p, 0);
    transform(c, p, w);
    wavespace(c, w, 0);
    c->nc = nc;
    free(p);
    double bmin = sqrt(c->b11);
    if (sqrt(c->b22) < bmin) bmin = sqrt(c->b22);
    if (sqrt(c->b33) < bmin) bmin = sqrt(c->b33);
    for (int k = 0; k < n / 2; k++) tk[k] = 0.;
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];
        double tf = x == 0 ? 1. : 2.;
        for (int y = 0; y < n; y++) {
            if (!mask_ok(c, a, y)) continue;
            size_t o = (size_t)a * n + y;
            double ksq = c->b11 * c->kx[x] * c->kx[x] + c->b22 * c->ky[y] * c->ky[y] + c->b33 * c->kz[z] * c->kz[z];
            int ik = (int)(sqrt(ksq) / bmin + 1.5);
            if (ik < 1 || ik > n / 2) continue;
            double term = 0.;
            for (int i = 0; i < 3; i++) term += c->un[i * vs + o].re * w[i * vs + o].re + c->un[i * vs + o].im * w[i * vs + o].im;
            tk[ik - 1] += term * tf;
        }
    }
    free(w);
    c->dt2 = dt2;
    double g6b[6] = {save[0][0], save[0][1], save[1][0], save[1][1], save[2][0], save[2][1]};
    orc_set_shifts(c, g6b);
}

/* vgmomt.f:50-143 (itransform.f:222-230, :385): moments of order 1..8 of
 * du/dx and dw/dz on the grid shifted by gsh[3] (the stage-1 shifts of an I/O
 * step), of u (which = 0) or un (which = 1), each sum divided by n^3.
 * out[0..7] = du/dx, out[8..15] = dw/dz.  The derivative factors are applied
 * in the z pencils as the reference does (itransform's nv = 6 path). */
void orc_gradient_moments(orc_ctx *c, int which, const double *gsh, double *out)
{
    int n = c->n, tot = c->xz_tot;
    size_t vs = (size_t)tot * n, np = (size_t)n * n * n;
    double save[3][2];
    memcpy(save, c->gsh, sizeof save);
    double g6[6] = {gsh[0], 0., gsh[1], 0., gsh[2], 0.};
    orc_set_shifts(c, g6);
    const cx *src = which == 0 ? c->u : c->un;
    cx *w = (cx *)calloc(6 * vs, sizeof(cx));
    memcpy(w + 4 * vs, src, sizeof(cx) * vs);             /* u -> x gradient slot */
    memcpy(w + 5 * vs, src + 2 * vs, sizeof(cx) * vs);    /* w -> z gradient slot */
    phase_shift(c, w, 6, 0);
    double *p = (double *)malloc(sizeof(double) * 6 * np);
    itransform(c, w, 6, p);
    for (int f = 0; f < 2; f++) {
        const double *g = p + (size_t)(4 + f) * np;
        double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (size_t i = 0; i < np; i++) {
            double v = g[i], sq = v * v;
            s[0] += v; s[1] += sq; s[2] += sq * v; s[3] += sq * sq;
            s[4] += sq * sq * v; s[5] += sq * sq * sq; s[6] += sq * sq * sq * v; s[7] += sq * sq * sq * sq;
        }
        for (int m = 0; m < 8; m++) out[8 * f + m] = s[m] / (double)np;
    }
    free(p);
    free(w);
    double g6b[6] = {save[0][0], save[0][1], save[1][0], save[1][1], save[2][0], save[2][1]};
    orc_set_shifts(c, g6b);
}

/* Piecewise hooks for tests: the inverse transform of u (3 vars) into
 * physical space p[3][y][z][x] (after the phase shift of stage kstep). */
void orc_itransform_only(orc_ctx *c, int kstep, const double *ucyl, double *p)
{
    size_t vs = (size_t)c->xz_tot * c->n;
    cx *w = (cx *)malloc(sizeof(cx) * 3 * vs);
    memcpy(w, ucyl, sizeof(cx) * 3 * vs);
    phase_shift(c, w, 3, kstep - 1);
    itransform(c, w, 3, p);
    free(w);
}

void orc_set_threads(int nt)
{
#ifdef _OPENMP
    omp_set_num_threads(nt);
#else
    (void)nt;
#endif
}

int orc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Initial field: homogeneous/field.f:169-257 (random solenoidal field, the  */
/* branch that draws its phases from ranu) followed by the conjugate        */
/* symmetry of homogeneous/consym.f:35-73 (FRESH, single task).  The        */
/* spectrum is E(k) = c0 k^4 exp(-2 (k/3)^2), c0 = 4/(sqrt(pi) 4.5^2.5), so */
/* that the continuous integral of E is 3/2 (u' = 1).                       */
/* ------------------------------------------------------------------------ */
static double espec(double k)
{
    double c0 = 4.0 / (sqrt(M_PI) * pow(4.5, 2.5));
    double q = k / 3.0;
    return c0 * k * k * k * k * exp(-2.0 * q * q);
}

void orc_field_init(orc_ctx *c, int seed, double *out /* [3][xz_tot][n] complex */)
{
    int n = c->n, tot = c->xz_tot;
    size_t vs = (size_t)tot * n;
    cx *u = (cx *)out;
    memset(u, 0, sizeof(cx) * 3 * vs);
    orc_rng r; rng_init(&r, seed); rng_ranseq(&r, 1);
    double pi = 4. * atan(1.);
    double voljac = 1.0 * 1.0 * 1.0;   /* beta1*beta2*beta3 with unit box */
    double twopi = 2. * pi;
    double rpid = 1. / sqrt(twopi);
    double s1 = sqrt(c->b11), s2 = sqrt(c->b22), s3 = sqrt(c->b33);
    voljac = s1 * s2 * s3;
    double s1d = 1. / s1, s2d = 1. / s2, s3d = 1. / s3;
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];
        double k1u = s1 * c->kx[x];
        double k3u = s3 * c->kz[z];
        int yst = (a == 0) ? 1 : 0;
        for (int y = yst; y < n; y++) {
            if (!mask_ok(c, a, y)) continue;
            double k2u = s2 * c->ky[y];
            double kyzsq = k2u * k2u + k3u * k3u;
            double k = sqrt(k1u * k1u + kyzsq);
            double kd = 1. / k;
            double ekx = espec(k) * voljac;
            double ef = sqrt(ekx) * rpid * kd;
            double theta1 = rng_ranu(&r);
            double theta2 = rng_ranu(&r);
            double phi = rng_ranu(&r);
            double k12 = sqrt(k1u * k1u + k2u * k2u);
            double angphi = twopi * phi;
            double t1 = twopi * theta1, t2 = twopi * theta2;
            cx e1 = cmk(cos(t1), sin(t1)), e2 = cmk(cos(t2), sin(t2));
            cx alpha = cscale(cos(angphi), cscale(ef, e1));
            cx beta = cscale(sin(angphi), cscale(ef, e2));
            size_t o = (size_t)a * n + y;
            if (k12 == 0.) {
                u[o] = cscale(1.0 / s1, alpha);
                u[o] = cmk(alpha.re / s1, alpha.im / s1);
                u[vs + o] = cmk(beta.re / s2, beta.im / s2);
                u[2 * vs + o] = CZERO;
            } else {
                cx ctmp1 = cscale(k, alpha);
                cx ctmp2 = cscale(k3u, beta);
                double rtmp = kd / k12;
                u[o] = cscale(s1d, cscale(rtmp, cadd(cscale(k2u, ctmp1), cscale(k1u, ctmp2))));
                u[vs + o] = cscale(s2d, cscale(rtmp, csub(cscale(k2u, ctmp2), cscale(k1u, ctmp1))));
                cx b3 = cscale(s3d, cscale(kd, cscale(k12, beta)));
                u[2 * vs + o] = cmk(-b3.re, -b3.im);
            }
        }
    }
    for (int i = 0; i < 3; i++) u[i * vs] = CZERO;
    /* consym (FRESH): kx = 0 plane */
    int kc0 = c->kc[0];
    for (int i = 0; i < 3; i++) {
        cx *ui = u + i * vs;
        ui[0] = cmk(ui[0].re, 0.);
        for (int y = n / 2 + 1; y < n; y++) ui[y] = cconj(ui[n - y]);
        for (int j = kc0 + 1; j < 2 * kc0 + 1; j++) {
            /* column j holds kz = j - (2 kc0 + 1) < 0; its mirror holds -kz */
            int kz = j - (2 * kc0 + 1);
            int jo = -kz;
            ui[(size_t)j * n + 0] = cconj(ui[(size_t)jo * n + 0]);
            for (int y = 1; y < n; y++) ui[(size_t)j * n + y] = cconj(ui[(size_t)jo * n + (n - y)]);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Shell spectra: homogeneous/sptr.f:139-193 (sums), :235-237 (2 nu),       */
/* :350-400 (ek, dk, tke, epslon, skew, Kolmogorov scales, integral scale). */
/* which = 0: u, 1: un.  ek, dk: [n]; stats: [7].                           */
/* ------------------------------------------------------------------------ */
void orc_spectra(orc_ctx *c, int which, double *ek, double *dk, double *eijk, double *stats)
{
    int n = c->n, tot = c->xz_tot, ns = n;
    size_t vs = (size_t)tot * n;
    const cx *u = which == 0 ? c->u : c->un;
    double *e6 = (double *)calloc((size_t)ns * 6, sizeof(double));
    double *d1 = (double *)calloc((size_t)ns, sizeof(double));
    double *s1 = (double *)calloc((size_t)ns, sizeof(double));
    double *ekk = (double *)calloc((size_t)ns, sizeof(double));
    for (int a = 0; a < tot; a++) {
        int x = c->ax[a], z = c->az[a];
        double tfact = (x == 0) ? 1. : 2.;
        for (int y = 0; y < n; y++) {
            if (!mask_ok(c, a, y)) continue;
            double kx2 = c->b11 * c->kx[x] * c->kx[x];
            double ky2 = (y == n / 2) ? 0. : c->b22 * c->ky[y] * c->ky[y];
            double kz2 = (z == n / 2) ? 0. : c->b33 * c->kz[z] * c->kz[z];
            double rk2 = kx2 + ky2 + kz2;
            int ik = (int)(sqrt(rk2) + 1.5);
            if (ik > ns) continue;
            cx v[3];
            for (int i = 0; i < 3; i++) v[i] = u[i * vs + (size_t)a * n + y];
            int ij = 0;
            for (int i = 0; i < 3; i++)
                for (int j = i; j < 3; j++) {
                    double uiuj = v[i].re * v[j].re + v[i].im * v[j].im;
                    double term = tfact * uiuj;
                    e6[(ik - 1) * 6 + ij] += term;
                    if (i == j) {
                        d1[ik - 1] += rk2 * term;
                        s1[ik - 1] += rk2 * term * rk2;
                        double ssq = i == 0 ? c->b11 : (i == 1 ? c->b22 : c->b33);
                        if (rk2 != 0.) ekk[ik - 1] += term / sqrt(rk2) * ssq;
                    }
                    ij++;
                }
        }
    }
    double nu = c->viscos, tke = 0, eps = 0, skew = 0, ekl = 0;
    for (int k = 0; k < ns; k++) {
        double e = (e6[k * 6 + 0] + e6[k * 6 + 3] + e6[k * 6 + 5]) * 0.5;
        double d = (2 * nu * d1[k]) * 0.5;
        double sk = (2 * nu * s1[k]) * 0.5;
        if (k == 0) { e = 0; d = 0; }
        if (ek) ek[k] = e;
        if (dk) dk[k] = d;
        if (eijk) for (int j = 0; j < 6; j++) eijk[k * 6 + j] = e6[k * 6 + j];
        tke += e; eps += d; skew += sk;
        if (k < n / 2) ekl += ekk[k] / 2.;
    }
    double pi = 4. * atan(1.), klen = 0, kvel = 0, ktime = 0;
    if (eps > 0) {
        skew = 2. / 35. * pow(15. * nu / eps, 1.5) * skew;
        klen = pow(nu * nu * nu / eps, .25);
        kvel = pow(nu * eps, .25);
        ktime = pow(nu / eps, .5);
    }
    ekl = 1.5 * pi / (2 * tke) * ekl;
    if (stats) {
        stats[0] = tke; stats[1] = eps; stats[2] = skew; stats[3] = klen; stats[4] = kvel; stats[5] = ktime;
        stats[6] = ekl;
    }
    free(e6); free(d1); free(s1); free(ekk);
}
