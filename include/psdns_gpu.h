/*
 * psdns_gpu.h -- C-ABI of libpsdns_gpu, the B200 (sm_100a) implementation of
 * the PSDNS RK2 time-step hot path.
 *
 * The reference exposes no plugin API: one RK stage is the sequence of
 * Fortran calls in rksubstep (PSDNS/timestep_module.f:152-318) operating on
 * module globals (PSDNS/module.f:324-385), and one time step is the call
 * `call timestep()` at PSDNS/main.f:463 preceded by `call shifts` at
 * PSDNS/main.f:409.  Each entry point below names the reference routine(s)
 * it replaces.
 *
 * Conventions (Fortran iso_c_binding friendly):
 *  - every function returns int status: 0 = ok, nonzero = error; the
 *    message is available from psdns_gpu_last_error();
 *  - nothing aborts or traps; device-side failures set a status word;
 *  - scalars that the driver may want to pass by reference are pointers;
 *  - arrays are plain pointers with explicit sizes; complex data is
 *    interleaved (re, im) doubles, i.e. Fortran complex(8);
 *  - host buffers are borrowed for the duration of the call only; the
 *    library owns all device memory.
 *  - one host thread per context; one CUDA stream per context.
 */
#ifndef PSDNS_GPU_H
#define PSDNS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Precision of the device state and of the bulk FFT arithmetic. */
#define PSDNS_PREC_FP32 0
#define PSDNS_PREC_FP64 1

/* 1-D transform arithmetic of the stage kernels (psdns_params.dft). */
#define PSDNS_DFT_FP32 0
#define PSDNS_DFT_TC_BF16X3 1

/* State layouts for set/get.
 * PSDNS_LAYOUT_YCYL: the reference's y-cylinder array uy(ny,num_al,nv) of a
 *   single rank (jproc = 1), column-major: element (y, a, v) at
 *   ((v*xz_tot + a)*ny + y); a enumerates the (kx,kz) columns inside the
 *   truncation cylinder in the order of next_xz (PSDNS/mpisetup.f:710-732). */
#define PSDNS_LAYOUT_YCYL 0
/* PSDNS_LAYOUT_FULL: the whole half-complex spectrum u(nxh,ny,nz,nv),
 *   nxh = nx/2+1, column-major: element (x, y, z, v) at
 *   (((v*nz + z)*ny + y)*nxh + x) -- the shape FFTW's real-to-complex
 *   transform gives a real (nx,ny,nz) array (PSDNS/epfftw.f).  set_state
 *   keeps the modes inside the truncation cylinder (kx < kxn, |kz| <= kc(kx),
 *   PSDNS/mpisetup.f:307-357); get_state writes zeros outside it. */
#define PSDNS_LAYOUT_FULL 1

/* Which field get_state returns. */
#define PSDNS_FIELD_U  0   /* u  (module comp, PSDNS/module.f:324-385) */
#define PSDNS_FIELD_UN 1   /* un */

typedef struct psdns_params {
    int32_t nx, ny, nz;      /* grid; cubic boxes (nx = ny = nz), nx even */
    int32_t nc;              /* passive scalars (0 or 1)                     */
    int32_t precision;       /* PSDNS_PREC_FP32 or PSDNS_PREC_FP64           */
    int32_t kshift;          /* 1..4, PSDNS/shifts.f:7-26                    */
    int32_t ksran;           /* RNG sequence for shifts (PSDNS/input.f:269)  */
    int32_t seed_input;      /* iseed record of the input file               */
    int32_t kranf1, kranf2;  /* RNG sequences for forcing (PSDNS/input.f:268)*/
    int32_t dft;             /* 1-D transforms: PSDNS_DFT_FP32 (Stockham
                                passes in the state precision) or
                                PSDNS_DFT_TC_BF16X3 (tensor cores, split BF16,
                                FP32 state at n = 1024 only)                */
    int32_t rkmethod;        /* 2 (proc4a/proc4b) or 4 (advanc_1..4, nc = 0,
                                no particles); 0 means 2 (PSDNS/input.f:222) */
    int32_t reserved_i[4];
    double viscos;           /* kinematic viscosity                          */
    double beta1, beta2, beta3; /* box scaling; 1 for a 2*pi box             */
    double cfl;              /* > 0: dt = cfl/velmax (PSDNS/step.f:77-78)    */
    double dt;               /* fixed time step when cfl <= 0                */
    double kforce;           /* Eswaran-Pope forcing radius; 0 = unforced    */
    double tforce, epsfor, tfiuo; /* forcing parameters (PSDNS/force.f:20-27) */
    double pr;               /* Schmidt number of the scalar                 */
    double grad[3];          /* mean scalar gradient                         */
    double reserved_d[8];
} psdns_params;

/* Fill *p with the reference's defaults (PSDNS/input and PSDNS/input.f). */
int psdns_gpu_default_params(psdns_params *p);

/* Truncation-cylinder geometry for an n^3 box (PSDNS/mpisetup.f:307-357):
 * number of kx columns kept (max_al_x), xz_tot, and optionally cut_z(x)
 * (array of *kxn ints) and the column start offsets (array of *kxn+1). */
int psdns_gpu_geometry(int32_t n, int32_t *kxn, int32_t *xz_tot,
                       int32_t *cut_z, int32_t *colstart);

/* The spherical mask of that geometry (PSDNS/masks.f:46-83) as the largest
 * kept |ky| per cylinder column: entry y of column a is inside when
 * y != n/2 and min(y, n-y) <= kymax[a] (array of xz_tot ints). */
int psdns_gpu_kymax(int32_t n, int32_t *kymax);

/* Create a context: validate parameters, build the cylinder map and the
 * spherical mask (PSDNS/masks.f), allocate the device state and work
 * arrays, and build twiddle tables.  Replaces the set-up calls of
 * PSDNS/main.f:160-286 (param_set, mpisetup, mpisetup2, epfftw, masks). */
int psdns_gpu_init(const psdns_params *p, void **ctx);

/* Release the context (and its device memory).  Replaces the end of main. */
int psdns_gpu_finalize(void *ctx);

/* Load the velocity state un (and u = un, PSDNS/incond.f:146) from a host
 * array in the given layout (complex(8), 3+nc variables). */
int psdns_gpu_set_state(void *ctx, const double *un, int32_t layout);

/* Random solenoidal initial field on the device, un = u (replaces
 * PSDNS/homogeneous/field.f:169-257 with PSDNS/homogeneous/consym.f:35-73,
 * the ranu-phase branch).  Spectrum E(k) = c0 k^4 exp(-2 (k/3)^2) with
 * integral 3/2 (u' = 1); seed starts the ranu stream (PSDNS/ranu.f). */
int psdns_gpu_field_init(void *ctx, int32_t seed);

/* The sinusoidal initial field of the shipped example runs, kinit(1) = -2
 * (replaces PSDNS/incond.f:196-209 -> inpvf.f:26-57 -> the hook
 * PSDNS/hooks/initial_conditions/pfield.f): u = au sin x cos y cos z,
 * v = av cos x sin y cos z, w = -(au + av) cos x cos y sin z (pfield uses
 * au = av = 1), transformed with the 1/n^3 forward normalisation; un = u,
 * other variables zero.  The reference requires zero shifts (kshift = 4)
 * with this field. */
int psdns_gpu_field_sinusoidal(void *ctx, double au, double av);

/* Copy u or un back to a host array (complex(8), 3+nc variables). */
int psdns_gpu_get_state(void *ctx, double *out, int32_t which, int32_t layout);

/* Asynchronous versions of set_state/get_state (PSDNS_LAYOUT_YCYL only):
 * the copies run on the context's own copy streams through device staging
 * (2 x 16 bytes per state element, allocated on first use), in chunks that
 * overlap the conversions, and an upload overlaps the download issued before
 * it (PCIe is full duplex).  Work on the state issued afterwards (step,
 * rk_stage, spectra, ...) is ordered after the upload.  The host buffers
 * must stay untouched until psdns_gpu_sync returns; an upload from the host
 * range of a pending download reads each chunk after it has landed. */
int psdns_gpu_set_state_async(void *ctx, const double *un, int32_t layout);
int psdns_gpu_get_state_async(void *ctx, double *out, int32_t which, int32_t layout);
/* Asynchronous copies of the entries inside the truncation sphere only
 * (PSDNS_LAYOUT_YCYL; the mask of PSDNS/masks.f:46-83: y != ny/2 and
 * min(y, ny-y) <= kymax of the column).  These are the entries the step
 * reads and writes: the reference updates un only inside the mask
 * (PSDNS/homogeneous/proc4b.f:183-191), so the others keep their values.
 * The host array must be pinned (cudaHostAlloc or cudaHostRegister): kernels
 * read or write it directly over the bus, 63% of the bytes of the full
 * array, with no device staging.  Entries outside the sphere are neither
 * read nor written.  An upload issued right after a download of the same
 * array overlaps it chunk by chunk; work on the state issued afterwards is
 * ordered after the upload, and any other call first waits for a pending
 * download.  The host array must stay untouched until psdns_gpu_sync. */
int psdns_gpu_set_state_sphere_async(void *ctx, const double *un);
/* Pin (page-lock and map) an existing host array for the sphere copies, and
 * undo it: a Fortran driver's uy array can then be passed as it is, without
 * calling the CUDA runtime itself.  Pinning is slow (do it once) and the
 * array must stay allocated until it is unpinned. */
int psdns_gpu_host_register(void *ptr, size_t bytes);
int psdns_gpu_host_unregister(void *ptr);
int psdns_gpu_get_state_sphere_async(void *ctx, double *out, int32_t which);
/* Wait for every copy and kernel of the context. */
int psdns_gpu_sync(void *ctx);

/* One full RK2 time step: shifts (PSDNS/shifts.f), then rksubstep(1) and
 * rksubstep(2) (PSDNS/timestep_module.f:25-55) with step/force at stage 1.
 * On return info[0..7] = dt, time, velmax, courant number, gsh(1..3,1)
 * (predictor shifts; info may be NULL). */
int psdns_gpu_step(void *ctx, double *info);

/* One RK stage with caller-supplied shifts and time step (the Fortran
 * driver keeps control of dt, PSDNS/timestep_module.f:70-481):
 * kstep = 1 or 2; gsh = gsh(3,2) column-major (PSDNS/shifts.f);
 * dt = time step (stage 1; ignored at stage 2, which reuses stage 1's);
 * velmax_out (stage 1) receives max N(|u|+|v|+|w|) (PSDNS/realspace_vel.f:108-110).
 * forcing may be NULL (unforced); otherwise for(kfor,k2fo,k2fo,3) complex(8)
 * (PSDNS/force.f:115-161). */
int psdns_gpu_rk_stage(void *ctx, int32_t kstep, const double *gsh, const double *dt,
                       const double *forcing, double *velmax_out);

/* Lagrangian particles (replaces the LAG_LOCAL hooks: partin positions in,
 * partsp.f RK2 with spcal_local.f cubic-spline interpolation).  pos is
 * column-major (np,3) = pp(np,1:3): FP64 positions in grid units, grid plane
 * i (1-based) at 1 + (i-1) + gsh(.,1) (PSDNS/hooks/LAG_LOCAL/partsp.f:44-51).
 * Each psdns_gpu_step then advances them at stage 1 with the spline of the
 * stage-1 velocity field, lagging the Eulerian field by one step
 * (partsp.f:231-299,405-412); the first step only interpolates velocities.
 * set replaces any previous particles; np = 0 removes them. */
int psdns_gpu_particles_set(void *ctx, int64_t np, const double *pos);

/* Positions pp(np,1:3) and velocities pp(np,4:6), column-major (np,3) each
 * (either may be NULL). */
int psdns_gpu_particles_get(void *ctx, double *pos, double *vel);
/* Particle output of one writing task (hooks/LAG_LOCAL/lagout1.f ->
 * pop1_file_local.f + pop1_write_local2.f with nsubset = 1): particles
 * ordered as the reference's tetrad groups, np = nrefp (1 + 3 ngp) (the
 * reference particles, then for each group three satellite sets).  Files
 * <prefix>/<igp>/pvel1g<igp>_s0 and .../ppos1g<igp>_s0 (directories made by
 * the caller), big-endian unformatted; append = 0 starts them with the
 * record (4 nrefp, nrefp, 4, 3); each call adds (istep - 1, time) and, per
 * component, the reference set and the group's three satellite sets. */
int psdns_gpu_particles_write(void *ctx, const char *prefix, int32_t ngp, int32_t istep, int32_t append);

/* The particle phase of psdns_gpu_step for a driver that runs the stages
 * itself with psdns_gpu_rk_stage: call it before rk_stage(kstep = 1) of each
 * step (partsp.f is called at the start of rksubstep(1),
 * PSDNS/timestep_module.f:168-186), with that stage's shifts gsh(1:3,1) and
 * the previous step's dt (rk_advpos.f:31-37; ignored by the first call, which
 * only interpolates).  Builds the spline of the current un on the shifted
 * grid and advances the particles (partin.f positions from
 * psdns_gpu_particles_init are made here too). */
int psdns_gpu_particles_advance(void *ctx, const double *gsh1, double dt_prev);

/* Shell spectra in FP64 (replaces PSDNS/homogeneous/sptr.f:139-400 for the
 * velocity): shells ik = int(|k| + 1.5), n of them (mxyz, comsp_set.f:14).
 * which = PSDNS_FIELD_UN (as sptr(un,...)) or PSDNS_FIELD_U.  Outputs (each
 * may be NULL): ek[n] = E(k), dk[n] = D(k) (2 nu k^2 E, shell 1 zeroed as in
 * sptr.f:355-357), eijk[n*6] = sum tfact Re(u_i u_j*) per shell for ij = 11,
 * 12, 13, 22, 23, 33, stats[7] = tke, epsilon, skewness (sptr.f:365),
 * Kolmogorov length, velocity and time, integral scale (sptr.f:387-390). */
int psdns_gpu_spectra(void *ctx, int32_t which, double *ek, double *dk, double *eijk, double *stats);

/* Eswaran-Pope forcing diagnostics of the last step (PSDNS/forcdt.f:18-41):
 * efk[kfor] energy input per shell, eirate[3] per component, *erate total
 * (each pointer may be NULL).  Error if the context is unforced. */
int psdns_gpu_forcing_stats(void *ctx, double *efk, double *eirate, double *erate);

/* The forcing table for(kfor,k2fo,k2fo,3) (complex(8), PSDNS/force.f:115-161)
 * used by the last step, and its dimensions (param_set.f:33,37). */
int psdns_gpu_forcing_table(void *ctx, double *table, int32_t *kfor, int32_t *k2fo);

/* Run statistics: time, dt, velmax, jstep. */
int psdns_gpu_get_time(void *ctx, double *out4);

/* The CUDA stream (cudaStream_t) on which the context launches all its work,
 * so that a caller can time or order work against it.  Plumbing; no
 * counterpart in the reference. */
int psdns_gpu_get_stream(void *ctx, void **stream);

/* Per-kernel device timing with CUDA events on the context's stream
 * (replaces the MPI_WTIME stage timers tt(1..10) of
 * PSDNS/timestep_module.f:90-478).  enable != 0 starts (and zeroes) the
 * accumulation; psdns_gpu_kernel_times returns, for the five stage kernels
 * (y backward, z backward, x chain, z forward, y forward + update) and the
 * particle phase (spline transform + particle step, 4 launches), the summed
 * milliseconds ms[6] and counts launches[6]. */
int psdns_gpu_profile(void *ctx, int32_t enable);
int psdns_gpu_kernel_times(void *ctx, double *ms, int64_t *launches);

/* Learned coarse solver.  No counterpart in the reference, which runs the
 * resolved DNS only; judged on the reference's statistics (E(k), epsilon
 * and skewness of PSDNS/homogeneous/sptr.f:354-365, du/dx moments of
 * PSDNS/vgmomt.f).  A coarse box advanced by psdns_gpu_step is corrected
 * after each step by a per-shell eddy viscosity nu_t(k) = nu g(k), g the
 * output of a spectral-correction network (4 layers: features -> width ->
 * width -> width -> 1, tanh, softplus output; BF16 weights, FP32
 * accumulation) from per-shell features of the box's spectrum.
 *
 * psdns_gpu_filter_state: the coarse box's u and un become the fine box's
 *   un restricted to the coarse truncation sphere (sharp filter in
 *   wavenumber space), both boxes in the same precision on this device.
 * psdns_gpu_shell_factor: multiply u and un of every mode of shell
 *   int(|k| + 0.5) = i, 1 <= i <= nshell, by f[i] (f[0..nshell]).
 * psdns_gpu_corrector_features: features of shells 1..nshell of u or un:
 *   x[3 (i-1) + 0..2] = i / kmax, log10(E(i) i^(5/3) / eps^(2/3)) (clamped
 *   to +-10), log10(kmax eta) with eps the resolved dissipation.
 * psdns_gpu_corrector_apply: features of un for the resolved shells, network
 *   forward pass, damping exp(-nu g(i) i^2 dt) with the last step's dt;
 *   info[0] = 1 if applied, 0 if the plain step was kept (non-finite,
 *   negative or runaway output: the fallback); info[1] = max g.
 * psdns_gpu_corrector_create/destroy: a network with Glorot-uniform weights
 *   from seed.  _params: get (get != 0) or set the PSDNS_CORRECTOR_PARAMS
 *   FP32 master weights (W0[H][F] b0 W1[H][H] b1 W2[H][H] b2 W3[H] b3).
 *   _forward: g for nb feature rows.  _grad: for the loss
 *   L = sum w (a g - tau)^2 / sum w over nb samples, its value and its
 *   gradient with respect to the master weights (forward with the BF16
 *   weights).  _train: iters full-batch Adam steps (learning rate lr) on the
 *   device; loss_hist[iters] (may be NULL) gets the loss before each step. */
#define PSDNS_CORRECTOR_FEATURES 3
#define PSDNS_CORRECTOR_WIDTH 32
#define PSDNS_CORRECTOR_PARAMS 2273
int psdns_gpu_filter_state(const void *fine, void *coarse);
int psdns_gpu_shell_factor(void *ctx, int32_t nshell, const double *f);
int psdns_gpu_corrector_features(void *ctx, int32_t which, int32_t nshell, float *x);
int psdns_gpu_corrector_apply(void *corr, void *ctx, double *info);
int psdns_gpu_corrector_create(int32_t seed, void **corr);
int psdns_gpu_corrector_destroy(void *corr);
int psdns_gpu_corrector_params(void *corr, int32_t get, float *w);
int psdns_gpu_corrector_forward(void *corr, int64_t nb, const float *x, float *g);
int psdns_gpu_corrector_grad(void *corr, int64_t nb, const float *x, const float *a, const float *tau,
                             const float *wt, float *grad, double *loss);
int psdns_gpu_corrector_train(void *corr, int64_t nb, const float *x, const float *a, const float *tau,
                              const float *wt, int32_t iters, double lr, double *loss_hist);

/* Batched forward 1-D DFT of nlines lines of n = 1024 complex points,
 * X_k = sum_j x_j exp(-2 pi i jk/n): the transform the stage kernels run
 * along every axis (the reference's FFTW 1-D transforms planned in
 * PSDNS/epfftw.f, e.g. PSDNS/transform.f:134).  mode 0: FP32 Stockham
 * radix-32 passes; mode 1: tensor cores (tcgen05.mma), split-BF16 operands
 * (hi + lo, three products) with FP32 accumulation.  in/out: host complex(8)
 * arrays of nlines*n values (computed in FP32).  A standalone check and
 * comparison of the two DFT forms; it allocates its own device buffers. */
int psdns_gpu_dft_lines(int32_t n, int64_t nlines, int32_t mode, const double *in, double *out);

/* Diagnostic of the tensor-core operand layouts: d = a b^T for a (128 x 64,
 * row-major) and b (64 x 64, row-major: row n holds column n of b^T),
 * both rounded to BF16, with one tcgen05.mma tile accumulated in FP32;
 * a_mn_major selects the layout of a in shared memory (1: MN-major, as the
 * DFT uses, 0: K-major).  No counterpart in the reference. */
int psdns_gpu_tc_gemm_check(int32_t a_mn_major, const float *a, const float *b, float *d);

/* One RK stage that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc, such as a
 * Fortran/OpenACC driver whose device arrays belong to another runtime, or a
 * process with a fixed device-memory budget.  The caller passes its own device
 * arrays u and un (YCYL layout, 3 variables, complex float for
 * PSDNS_PREC_FP32 or complex double for PSDNS_PREC_FP64) on the current
 * device; all other device memory comes from one static array of
 * PSDNS_NOALLOC_BYTES per GPU, held until the process exits.  Boxes up to
 * PSDNS_NOALLOC_MAX_N^3 (16, 32 or 64), unforced, nc = 0; larger sizes are
 * rejected.  gsh = gsh(3,2) column-major; dt = the step's dt, passed at both
 * stages; velmax_out (stage 1) as in psdns_gpu_rk_stage; stream = a
 * cudaStream_t or NULL.  Each call looks up the array's device address,
 * copies its tables from host memory and synchronises the stream before it
 * returns; a stream that is being captured is refused with an error.  Calls
 * share the array, so calls that overlap on the GPU race.  Host pointers and
 * other devices' memory are rejected. */
#define PSDNS_NOALLOC_MAX_N 64
#define PSDNS_NOALLOC_BYTES (16u * 1024u * 1024u)
int psdns_gpu_rk_stage_noalloc(const psdns_params *p, int32_t kstep, const double *gsh, const double *dt,
                               void *u_dev, void *un_dev, double *velmax_out, void *stream);

/* ------------------------------------------------------------------------
 * Ensembles: independent boxes advanced together (no reference routine: the
 * reference runs one box per job).  p[0..count-1] describe the boxes; each
 * has its own grid size (16..1024 powers of two, 48, 96), viscosity, dt or
 * cfl, kshift and seed, and follows exactly the run of a single context made
 * with the same parameters.  All boxes share precision and beta; nc = 0,
 * kforce = 0.  Boxes of the same n share every kernel launch (the box is a
 * grid dimension); boxes with a fixed dt (cfl <= 0) replay each step from a
 * captured CUDA graph.
 * ------------------------------------------------------------------------ */
int psdns_gpu_ensemble_create(const psdns_params *p, int32_t count, void **ens);
int psdns_gpu_ensemble_destroy(void *ens);
/* Random solenoidal initial field of box i from seeds[i] (as psdns_gpu_field_init). */
int psdns_gpu_ensemble_field_init(void *ens, const int32_t *seeds);
/* State of one box (PSDNS_LAYOUT_YCYL, 3 variables). */
int psdns_gpu_ensemble_set_state(void *ens, int32_t box, const double *un, int32_t layout);
int psdns_gpu_ensemble_get_state(void *ens, int32_t box, double *out, int32_t which, int32_t layout);
/* nsteps RK2 steps of every box; info[8*i .. 8*i+7] = the last step's
 * psdns_gpu_step info of box i.  Returns 2 if a box met an abort condition
 * of step.f (the steps are completed). */
int psdns_gpu_ensemble_step(void *ens, int32_t nsteps, double *info);
/* The ensemble autotuner's choices (no reference routine; the counterpart
 * of FFTW's planner and wisdom, PSDNS/epfftw.f, PSDNS/wisdom.c): per class
 * of equal n, in the first steps of a fixed-dt class, the number of boxes
 * per launch, then the FFT tiles of the z transforms (x lines per block of
 * K2 and K4: the default, half, double; boxes of n <= 128), each candidate
 * timed over two real steps.  out[8 * cap] rows: n, boxes, tuned (0/1),
 * boxes per launch, K2 lines per block, K4 lines per block, step ms of the
 * all-default candidate, step ms of the choice; *nclasses = classes. */
int psdns_gpu_ensemble_tuning(void *ens, int32_t cap, double *out, int32_t *nclasses);
/* Shell spectra of one box (as psdns_gpu_spectra). */
int psdns_gpu_ensemble_spectra(void *ens, int32_t box, int32_t which, double *ek, double *dk, double *eijk,
                               double *stats);

/* Initial particle positions as partin (hooks/LAG_LOCAL/partin.f) makes
 * them, at the first particle phase of the next step (with that step's
 * stage-1 shifts): pstart = 0, nop uniform random positions, nearly equal
 * numbers per y-slice, from RNG sequence kipran (compart_set.f:160 sets 11);
 * pstart = -1, a cubic lattice of nop^3 grid nodes. */
int psdns_gpu_particles_init(void *ctx, int64_t nop, int32_t pstart, int32_t kipran);

/* Checkpoints in the reference's own file format: one task's pencil file
 * as homogeneous/outpen_write_r.f writes it (big-endian unformatted
 * records, real(8) pairs, kx = 0..nx/2-1, Nyquist y and z planes left out),
 * e.g. outpen/0/outpenc.p0.  write: u or un of the context; read: sets un
 * and u (modes outside the truncation cylinder are dropped).  path is a
 * NUL-terminated file name. */
/* Multi-task pencil sets (homogeneous/outpen_write_r.f, inpen_read_r.f):
 * write_checkpoint_set writes iproc*jproc files "<prefix>.p<t>", task
 * t = jp*iproc + ip holding x in [ip xisz, (ip+1) xisz) and z in
 * [jp zjsz, (jp+1) zjsz), xisz = (n/2)/iproc, zjsz = n/jproc, each in the
 * one-task file's record layout with its own xist/xisz/zjst/zjsz header;
 * read_checkpoint_set reads any set of such files (paths[nfiles]), placing
 * each pencil by its header, and checks that the set covers every (x, z)
 * of the box once. */
int psdns_gpu_write_checkpoint_set(void *ctx, const char *prefix, int32_t iproc, int32_t jproc, int32_t which);
int psdns_gpu_read_checkpoint_set(void *ctx, const char *const *paths, int32_t nfiles);
/* Checkpoint metadata.  write_chkptou: PSDNS/store.f icall 1 + 2 (called
 * at PSDNS/main.f:583): the integers nx ny nz my mz nxhvs nyvs nzvs nc ncd
 * kfor iostep kshift and istep (format 10i8; my..nzvs are never set by
 * store.f and are written as 0) and the reals viscos pr a11 a22 a33 shear
 * grad beta1-3 cfl dt tforce epsfor kforce tfiuo, then time gsh(:,2)
 * b11 b22 b33 b12 (2 each) and the forcing processes suo svo (format
 * 1p5e15.8).  read_chkptou: store.f icall 3 (incond.f:262): with strict,
 * the stored parameters must be this run's (kstop = 1, store.f:272-301);
 * restores time, gsh(:,2), suo and svo, returns istep in *istep, and makes
 * the next step the first of a restarted run (no initial shift draw,
 * shifts.f:47; forcing processes kept, vfuo.f/vfiuo.f with istart > 0).
 * write_ranout / read_ranin: the 20 RNG seeds of PSDNS/ranseq.f (k = -2,
 * :174-183, and k = -1, :83-118; format 5i15). */
int psdns_gpu_write_chkptou(void *ctx, const char *path, int32_t istep, int32_t iostep);
int psdns_gpu_read_chkptou(void *ctx, const char *path, int32_t strict, int32_t *istep);
int psdns_gpu_write_ranout(void *ctx, const char *path);
int psdns_gpu_read_ranin(void *ctx, const char *path);
int psdns_gpu_write_checkpoint(void *ctx, const char *path, int32_t which);
int psdns_gpu_read_checkpoint(void *ctx, const char *path);

/* Transfer spectrum (replaces homogeneous/trfsp.f, called at stage 1 of
 * I/O steps): tk[k-1] = sum over shell k = 1..nx/2 (int(|k|/min(beta) +
 * 1.5)) of tfact Re(conj(un) . N(u)), with N(u) the convective term
 * evaluated on the grid shifted by gsh[3] (the step's gsh(:,1); null =
 * unshifted).  FP64 sums; the state is not changed. */
int psdns_gpu_transfer_spectrum(void *ctx, const double *gsh, double *tk);

/* One-dimensional spectra and the length/time scales of sptr
 * (homogeneous/sptr.f:119-218, :311-468), FP64: xr, yr, zr [6][nx/2+1] are
 * the normalised spectra along x, y, z of the pairs 11,12,13,22,23,33;
 * stats[55] = corr[6], integral scales lijk[6][3], rms[3], integral-scale
 * Reynolds numbers raak[3], eddy turnover times ett[3], mean square
 * derivatives tmij[3][3] (component i, direction a), grdiss, Taylor
 * microscales taak[3][3], Taylor Reynolds numbers tmre[3].  Any output may
 * be null. */
int psdns_gpu_spectra_scales(void *ctx, int32_t which, double *xr, double *yr, double *zr, double *stats);

/* Moments of the velocity gradients (replaces PSDNS/vgmomt.f, called from
 * itransform.f:385 on I/O steps): out[0..7] = <(du/dx)^m>, m = 1..8, and
 * out[8..15] = <(dw/dz)^m> of u or un, averaged over the n^3 points of the
 * grid shifted by gsh[3] in grid units (the stage-1 shifts gsh(:,1) of the
 * step, as in the reference; null = unshifted).  FP64 sums. */
int psdns_gpu_gradient_moments(void *ctx, int32_t which, const double *gsh, double *out);

/* Message of the last error on this thread ("" if none). */
int psdns_gpu_last_error(char *buf, int32_t len);

#ifdef __cplusplus
}
#endif

#endif /* PSDNS_GPU_H */
