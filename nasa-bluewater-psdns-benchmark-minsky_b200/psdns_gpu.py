"""Python binding of libpsdns_gpu (the C-ABI declared in include/psdns_gpu.h).

The binding mirrors how the reference's Fortran driver would use the library:
`Solver(params)` replaces the set-up calls of PSDNS/main.f:160-286,
`set_state` replaces incond (PSDNS/incond.f), `step` replaces one pass of the
time loop (`call shifts` + `call timestep`, PSDNS/main.f:409-463) and
`rk_stage` replaces one `rksubstep` (PSDNS/timestep_module.f:70-481).

The library must be built (build.py) and a CUDA device present; there is no
CPU fallback: every method raises if the library or the device is missing.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "libpsdns_gpu.so")
_LIB = None

PREC_FP32 = 0
PREC_FP64 = 1
DFT_FP32 = 0          # psdns_params.dft: Stockham passes in the state precision
DFT_TC_BF16X3 = 1     # tensor cores, split-BF16 operands, FP32 accumulation (FP32 state, n = 1024)
LAYOUT_YCYL = 0
LAYOUT_FULL = 1
FIELD_U = 0
FIELD_UN = 1

# every entry point declared in include/psdns_gpu.h
EXPORTS = (
    "psdns_gpu_field_sinusoidal",
    "psdns_gpu_transfer_spectrum",
    "psdns_gpu_spectra_scales",
    "psdns_gpu_particles_init",
    "psdns_gpu_write_checkpoint",
    "psdns_gpu_read_checkpoint",
    "psdns_gpu_gradient_moments",
    "psdns_gpu_set_state_async",
    "psdns_gpu_set_state_sphere_async",
    "psdns_gpu_kymax",
    "psdns_gpu_particles_advance",
    "psdns_gpu_host_register",
    "psdns_gpu_host_unregister",
    "psdns_gpu_get_state_sphere_async",
    "psdns_gpu_get_state_async",
    "psdns_gpu_sync",
    "psdns_gpu_ensemble_create",
    "psdns_gpu_ensemble_destroy",
    "psdns_gpu_ensemble_field_init",
    "psdns_gpu_ensemble_set_state",
    "psdns_gpu_ensemble_get_state",
    "psdns_gpu_ensemble_step",
    "psdns_gpu_ensemble_tuning",
    "psdns_gpu_ensemble_spectra",
    "psdns_gpu_default_params",
    "psdns_gpu_geometry",
    "psdns_gpu_init",
    "psdns_gpu_finalize",
    "psdns_gpu_set_state",
    "psdns_gpu_get_state",
    "psdns_gpu_step",
    "psdns_gpu_rk_stage",
    "psdns_gpu_get_time",
    "psdns_gpu_last_error",
    "psdns_gpu_field_init",
    "psdns_gpu_get_stream",
    "psdns_gpu_profile",
    "psdns_gpu_kernel_times",
    "psdns_gpu_rk_stage_noalloc",
    "psdns_gpu_dft_lines",
    "psdns_gpu_filter_state",
    "psdns_gpu_particles_write",
    "psdns_gpu_write_checkpoint_set",
    "psdns_gpu_read_checkpoint_set",
    "psdns_gpu_write_chkptou",
    "psdns_gpu_read_chkptou",
    "psdns_gpu_write_ranout",
    "psdns_gpu_read_ranin",
    "psdns_gpu_shell_factor",
    "psdns_gpu_corrector_features",
    "psdns_gpu_corrector_apply",
    "psdns_gpu_corrector_create",
    "psdns_gpu_corrector_destroy",
    "psdns_gpu_corrector_params",
    "psdns_gpu_corrector_forward",
    "psdns_gpu_corrector_grad",
    "psdns_gpu_corrector_train",
    "psdns_gpu_tc_gemm_check",
    "psdns_gpu_forcing_stats",
    "psdns_gpu_spectra",
    "psdns_gpu_particles_set",
    "psdns_gpu_particles_get",
    "psdns_gpu_forcing_table",
)


class Params(ctypes.Structure):
    """psdns_params of include/psdns_gpu.h."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("nc", ctypes.c_int32), ("precision", ctypes.c_int32), ("kshift", ctypes.c_int32),
        ("ksran", ctypes.c_int32), ("seed_input", ctypes.c_int32),
        ("kranf1", ctypes.c_int32), ("kranf2", ctypes.c_int32),
        ("dft", ctypes.c_int32), ("rkmethod", ctypes.c_int32), ("reserved_i", ctypes.c_int32 * 4),
        ("viscos", ctypes.c_double), ("beta1", ctypes.c_double), ("beta2", ctypes.c_double),
        ("beta3", ctypes.c_double), ("cfl", ctypes.c_double), ("dt", ctypes.c_double),
        ("kforce", ctypes.c_double), ("tforce", ctypes.c_double), ("epsfor", ctypes.c_double),
        ("tfiuo", ctypes.c_double), ("pr", ctypes.c_double), ("grad", ctypes.c_double * 3),
        ("reserved_d", ctypes.c_double * 8),
    ]


class PsdnsError(RuntimeError):
    pass


def lib_path():
    return _LIBPATH


def load():
    """Load libpsdns_gpu.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(_LIBPATH):
        raise PsdnsError(f"{_LIBPATH} is missing: run build.py (there is no CPU fallback)")
    L = ctypes.CDLL(_LIBPATH)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
    L.psdns_gpu_default_params.argtypes = [ctypes.POINTER(Params)]
    L.psdns_gpu_geometry.argtypes = [ctypes.c_int32, ip, ip, ip, ip]
    L.psdns_gpu_kymax.argtypes = [ctypes.c_int32, ip]
    L.psdns_gpu_particles_advance.argtypes = [vp, dp, ctypes.c_double]
    L.psdns_gpu_host_register.argtypes = [vp, ctypes.c_size_t]
    L.psdns_gpu_host_unregister.argtypes = [vp]
    L.psdns_gpu_init.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p)]
    L.psdns_gpu_finalize.argtypes = [vp]
    L.psdns_gpu_set_state.argtypes = [vp, dp, ctypes.c_int32]
    L.psdns_gpu_get_state.argtypes = [vp, dp, ctypes.c_int32, ctypes.c_int32]
    L.psdns_gpu_step.argtypes = [vp, dp]
    L.psdns_gpu_rk_stage.argtypes = [vp, ctypes.c_int32, dp, dp, dp, dp]
    L.psdns_gpu_get_time.argtypes = [vp, dp]
    L.psdns_gpu_last_error.argtypes = [ctypes.c_char_p, ctypes.c_int32]
    L.psdns_gpu_field_init.argtypes = [vp, ctypes.c_int32]
    L.psdns_gpu_get_stream.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    L.psdns_gpu_profile.argtypes = [vp, ctypes.c_int32]
    L.psdns_gpu_kernel_times.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int64)]
    L.psdns_gpu_forcing_stats.argtypes = [vp, dp, dp, dp]
    L.psdns_gpu_particles_set.argtypes = [vp, ctypes.c_int64, dp]
    L.psdns_gpu_particles_get.argtypes = [vp, dp, dp]
    L.psdns_gpu_spectra.argtypes = [vp, ctypes.c_int32, dp, dp, dp, dp]
    L.psdns_gpu_forcing_table.argtypes = [vp, dp, ip, ip]
    L.psdns_gpu_rk_stage_noalloc.argtypes = [ctypes.POINTER(Params), ctypes.c_int32, dp, dp, vp, vp, dp, vp]
    L.psdns_gpu_filter_state.argtypes = [vp, vp]
    L.psdns_gpu_particles_write.argtypes = [vp, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    cp = ctypes.c_char_p
    L.psdns_gpu_write_checkpoint_set.argtypes = [vp, cp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.psdns_gpu_read_checkpoint_set.argtypes = [vp, ctypes.POINTER(cp), ctypes.c_int32]
    L.psdns_gpu_write_chkptou.argtypes = [vp, cp, ctypes.c_int32, ctypes.c_int32]
    L.psdns_gpu_read_chkptou.argtypes = [vp, cp, ctypes.c_int32, ip]
    L.psdns_gpu_write_ranout.argtypes = [vp, cp]
    L.psdns_gpu_read_ranin.argtypes = [vp, cp]
    L.psdns_gpu_shell_factor.argtypes = [vp, ctypes.c_int32, dp]
    fq = ctypes.POINTER(ctypes.c_float)
    L.psdns_gpu_corrector_features.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, fq]
    L.psdns_gpu_corrector_apply.argtypes = [vp, vp, dp]
    L.psdns_gpu_corrector_create.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
    L.psdns_gpu_corrector_destroy.argtypes = [vp]
    L.psdns_gpu_corrector_params.argtypes = [vp, ctypes.c_int32, fq]
    L.psdns_gpu_corrector_forward.argtypes = [vp, ctypes.c_int64, fq, fq]
    L.psdns_gpu_corrector_grad.argtypes = [vp, ctypes.c_int64, fq, fq, fq, fq, fq, dp]
    L.psdns_gpu_corrector_train.argtypes = [vp, ctypes.c_int64, fq, fq, fq, fq, ctypes.c_int32, ctypes.c_double, dp]
    L.psdns_gpu_dft_lines.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, dp, dp]
    fp = ctypes.POINTER(ctypes.c_float)
    L.psdns_gpu_tc_gemm_check.argtypes = [ctypes.c_int32, fp, fp, fp]
    L.psdns_gpu_field_sinusoidal.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    L.psdns_gpu_transfer_spectrum.argtypes = [vp, dp, dp]
    L.psdns_gpu_spectra_scales.argtypes = [vp, ctypes.c_int32, dp, dp, dp, dp]
    L.psdns_gpu_particles_init.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32]
    L.psdns_gpu_write_checkpoint.argtypes = [vp, ctypes.c_char_p, ctypes.c_int32]
    L.psdns_gpu_read_checkpoint.argtypes = [vp, ctypes.c_char_p]
    L.psdns_gpu_gradient_moments.argtypes = [vp, ctypes.c_int32, dp, dp]
    L.psdns_gpu_set_state_async.argtypes = [vp, dp, ctypes.c_int32]
    L.psdns_gpu_set_state_sphere_async.argtypes = [vp, dp]
    L.psdns_gpu_get_state_sphere_async.argtypes = [vp, dp, ctypes.c_int32]
    L.psdns_gpu_get_state_async.argtypes = [vp, dp, ctypes.c_int32, ctypes.c_int32]
    L.psdns_gpu_sync.argtypes = [vp]
    L.psdns_gpu_ensemble_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
    L.psdns_gpu_ensemble_destroy.argtypes = [vp]
    L.psdns_gpu_ensemble_field_init.argtypes = [vp, ip]
    L.psdns_gpu_ensemble_set_state.argtypes = [vp, ctypes.c_int32, dp, ctypes.c_int32]
    L.psdns_gpu_ensemble_get_state.argtypes = [vp, ctypes.c_int32, dp, ctypes.c_int32, ctypes.c_int32]
    L.psdns_gpu_ensemble_step.argtypes = [vp, ctypes.c_int32, dp]
    L.psdns_gpu_ensemble_tuning.argtypes = [vp, ctypes.c_int32, dp, ip]
    L.psdns_gpu_ensemble_spectra.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, dp, dp, dp, dp]
    for name in EXPORTS:
        getattr(L, name).restype = ctypes.c_int
    _LIB = L
    return L


def last_error():
    buf = ctypes.create_string_buffer(512)
    load().psdns_gpu_last_error(buf, 512)
    return buf.value.decode()


def _check(rc, what):
    if rc != 0:
        raise PsdnsError(f"{what} failed (status {rc}): {last_error()}")


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def default_params(**kw):
    p = Params()
    _check(load().psdns_gpu_default_params(ctypes.byref(p)), "psdns_gpu_default_params")
    for k, v in kw.items():
        if k == "n":
            p.nx = p.ny = p.nz = int(v)
        elif k == "grad":
            for i in range(3):
                p.grad[i] = float(v[i])
        else:
            setattr(p, k, v)
    return p


def geometry(n):
    kxn = ctypes.c_int32()
    tot = ctypes.c_int32()
    _check(load().psdns_gpu_geometry(n, ctypes.byref(kxn), ctypes.byref(tot), None, None), "geometry")
    cut = np.zeros(kxn.value, np.int32)
    col = np.zeros(kxn.value + 1, np.int32)
    ip = ctypes.POINTER(ctypes.c_int32)
    _check(load().psdns_gpu_geometry(n, None, None, cut.ctypes.data_as(ip), col.ctypes.data_as(ip)), "geometry")
    kym = np.zeros(tot.value, np.int32)
    _check(load().psdns_gpu_kymax(n, kym.ctypes.data_as(ip)), "kymax")
    return {"kxn": kxn.value, "xz_tot": tot.value, "cut": cut, "colstart": col, "kymax": kym}


def host_register(arr):
    """Pin a host numpy array in place (for the sphere copies); returns its address."""
    ptr = arr.ctypes.data
    _check(load().psdns_gpu_host_register(ctypes.c_void_p(ptr), arr.nbytes), "host_register")
    return ptr


def host_unregister(arr):
    _check(load().psdns_gpu_host_unregister(ctypes.c_void_p(arr.ctypes.data)), "host_unregister")


def sphere_mask(n):
    """[xz_tot, n] booleans: the entries inside the truncation sphere (masks.f)."""
    kym = geometry(n)["kymax"].astype(np.int64)
    y = np.arange(n)
    return (y[None, :] != n // 2) & (np.minimum(y, n - y)[None, :] <= kym[:, None])


def dft_lines(x, mode=DFT_TC_BF16X3):
    """Forward DFT along the last axis (1024 points) of a complex array on the
    device (psdns_gpu_dft_lines): mode DFT_FP32 (Stockham radix-32 passes)
    or DFT_TC_BF16X3 (tensor cores, split-BF16 operands, FP32 accumulation)."""
    a = np.ascontiguousarray(x, dtype=np.complex128)
    n = a.shape[-1]
    out = np.empty_like(a)
    _check(load().psdns_gpu_dft_lines(n, a.size // n, int(mode), _dp(a.view(np.float64)),
                                      _dp(out.view(np.float64))), "psdns_gpu_dft_lines")
    return out


def tc_gemm_check(a, b, a_mn_major=1):
    """d = a b^T on one tensor-core tile (a: 128 x 64, b: 64 x 64, rounded to BF16)."""
    fa = np.ascontiguousarray(a, dtype=np.float32)
    fb = np.ascontiguousarray(b, dtype=np.float32)
    d = np.zeros((128, 64), np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    _check(load().psdns_gpu_tc_gemm_check(int(a_mn_major), fa.ctypes.data_as(fp), fb.ctypes.data_as(fp),
                                          d.ctypes.data_as(fp)), "psdns_gpu_tc_gemm_check")
    return d


CORRECTOR_FEATURES = 3
CORRECTOR_WIDTH = 32
CORRECTOR_PARAMS = 2273


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def resolved_shells(n):
    """Shells 1..K of an n^3 box's truncation sphere: K = int(sqrt(2) n / 3 + 0.5)."""
    return int(np.sqrt(2.0) * n / 3.0 + 0.5)


class Corrector:
    """The spectral-correction network of the learned coarse solver
    (psdns_gpu_corrector_*): per-shell features -> eddy viscosity / nu."""

    def __init__(self, seed=1):
        h = ctypes.c_void_p()
        _check(load().psdns_gpu_corrector_create(int(seed), ctypes.byref(h)), "psdns_gpu_corrector_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            load().psdns_gpu_corrector_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def get_params(self):
        w = np.zeros(CORRECTOR_PARAMS, np.float32)
        _check(load().psdns_gpu_corrector_params(self._h, 1, _fp(w)), "corrector_params")
        return w

    def set_params(self, w):
        w = _f32(w)
        assert w.size == CORRECTOR_PARAMS
        _check(load().psdns_gpu_corrector_params(self._h, 0, _fp(w)), "corrector_params")

    def forward(self, x):
        x = _f32(x).reshape(-1, CORRECTOR_FEATURES)
        g = np.zeros(len(x), np.float32)
        _check(load().psdns_gpu_corrector_forward(self._h, len(x), _fp(x), _fp(g)), "corrector_forward")
        return g

    def grad(self, x, a, tau, wt):
        x = _f32(x).reshape(-1, CORRECTOR_FEATURES)
        a, tau, wt = _f32(a), _f32(tau), _f32(wt)
        g = np.zeros(CORRECTOR_PARAMS, np.float32)
        loss = np.zeros(1)
        _check(load().psdns_gpu_corrector_grad(self._h, len(x), _fp(x), _fp(a), _fp(tau), _fp(wt), _fp(g), _dp(loss)),
               "corrector_grad")
        return g, float(loss[0])

    def train(self, x, a, tau, wt, iters=2000, lr=3e-3):
        x = _f32(x).reshape(-1, CORRECTOR_FEATURES)
        a, tau, wt = _f32(a), _f32(tau), _f32(wt)
        hist = np.zeros(int(iters))
        _check(load().psdns_gpu_corrector_train(self._h, len(x), _fp(x), _fp(a), _fp(tau), _fp(wt), int(iters),
                                                float(lr), _dp(hist)), "corrector_train")
        return hist


NOALLOC_MAX_N = 64


def rk_stage_noalloc(params, kstep, gsh, dt, u_ptr, un_ptr, stream=0):
    """One RK stage on caller-owned device arrays with no device allocation
    (psdns_gpu_rk_stage_noalloc).  u_ptr/un_ptr: device addresses of the YCYL
    state in the params' precision; dt must be given at both stages.  Returns
    velmax at stage 1."""
    g = np.ascontiguousarray(np.asarray(gsh, np.float64).reshape(3, 2).T.reshape(-1))
    dtv = np.array([dt], np.float64)
    vm = np.zeros(1, np.float64)
    _check(load().psdns_gpu_rk_stage_noalloc(ctypes.byref(params), int(kstep), _dp(g), _dp(dtv),
                                             ctypes.c_void_p(u_ptr), ctypes.c_void_p(un_ptr), _dp(vm),
                                             ctypes.c_void_p(stream)),
           "psdns_gpu_rk_stage_noalloc")
    return vm[0]


class Solver:
    """One periodic box advanced on the GPU by the RK2 step of PSDNS."""

    def __init__(self, params=None, **kw):
        L = load()
        self.params = params if params is not None else default_params(**kw)
        self._ctx = ctypes.c_void_p()
        _check(L.psdns_gpu_init(ctypes.byref(self.params), ctypes.byref(self._ctx)), "psdns_gpu_init")
        self.n = self.params.nx
        self.nc = self.params.nc
        g = geometry(self.n)
        self.kxn = g["kxn"]
        self.xz_tot = g["xz_tot"]

    def close(self):
        if self._ctx:
            load().psdns_gpu_finalize(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def state_shape(self):
        """(3 + nc, xz_tot, n): velocity components, then the scalar."""
        return (3 + self.nc, self.xz_tot, self.n)

    def full_shape(self):
        """(3 + nc, nz, ny, nx/2+1): the Fortran array u(nxh,ny,nz,nv) in C order."""
        return (3 + self.nc, self.n, self.n, self.n // 2 + 1)

    def set_state(self, un, layout=LAYOUT_YCYL):
        a = np.ascontiguousarray(un, dtype=np.complex128)
        want = self.state_shape() if layout == LAYOUT_YCYL else self.full_shape()
        if a.shape != want:
            raise ValueError(f"state shape {a.shape} != {want}")
        _check(load().psdns_gpu_set_state(self._ctx, _dp(a.view(np.float64)), layout), "set_state")

    def set_state_ptr(self, ptr):
        """set_state from a raw host pointer (complex(8) YCYL, e.g. pinned memory)."""
        _check(load().psdns_gpu_set_state(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)),
                                          LAYOUT_YCYL), "set_state")

    def get_state(self, which=FIELD_UN, out=None, layout=LAYOUT_YCYL):
        if out is None:
            out = np.zeros(self.state_shape() if layout == LAYOUT_YCYL else self.full_shape(), np.complex128)
        _check(load().psdns_gpu_get_state(self._ctx, _dp(out.view(np.float64)), which, layout),
               "get_state")
        return out

    def set_state_async_ptr(self, ptr):
        """Upload from a pinned host pointer on the copy stream (returns at once)."""
        _check(load().psdns_gpu_set_state_async(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)),
                                                LAYOUT_YCYL), "set_state_async")

    def set_state_sphere_async_ptr(self, ptr):
        """Upload the entries inside the truncation sphere from pinned host memory (YCYL)."""
        _check(load().psdns_gpu_set_state_sphere_async(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double))),
               "set_state_sphere_async")

    def get_state_sphere_async_ptr(self, ptr, which=FIELD_UN):
        """Download the entries inside the truncation sphere to pinned host memory (YCYL)."""
        _check(load().psdns_gpu_get_state_sphere_async(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)),
                                                       which), "get_state_sphere_async")

    def get_state_async_ptr(self, ptr, which=FIELD_UN):
        """Download into a pinned host pointer on the copy stream (returns at once)."""
        _check(load().psdns_gpu_get_state_async(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)),
                                                which, LAYOUT_YCYL), "get_state_async")

    def sync(self):
        _check(load().psdns_gpu_sync(self._ctx), "sync")

    def get_state_ptr(self, ptr, which=FIELD_UN):
        _check(load().psdns_gpu_get_state(self._ctx, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)),
                                          which, LAYOUT_YCYL), "get_state")

    def step(self):
        info = np.zeros(8, np.float64)
        rc = load().psdns_gpu_step(self._ctx, _dp(info))
        if rc not in (0, 2):
            _check(rc, "psdns_gpu_step")
        return {"dt": info[0], "time": info[1], "velmax": info[2], "courant": info[3],
                "gsh1": info[4:7].copy(), "jstep": int(info[7]), "status": rc}

    def rk_stage(self, kstep, gsh, dt=None):
        g = np.ascontiguousarray(np.asarray(gsh, np.float64).reshape(3, 2).T.reshape(-1))
        dtv = np.array([dt if dt is not None else 0.0], np.float64)
        vm = np.zeros(1, np.float64)
        _check(load().psdns_gpu_rk_stage(self._ctx, int(kstep), _dp(g), _dp(dtv), None, _dp(vm)),
               "psdns_gpu_rk_stage")
        return vm[0]

    def field_init(self, seed):
        """Random solenoidal field (field.f restated) written to u and un on the device."""
        _check(load().psdns_gpu_field_init(self._ctx, int(seed)), "field_init")

    def field_sinusoidal(self, au=1.0, av=1.0):
        """pfield.f sinusoidal field u = au sin x cos y cos z, ..."""
        _check(load().psdns_gpu_field_sinusoidal(self._ctx, float(au), float(av)), "field_sinusoidal")

    def stream(self):
        """cudaStream_t (as int) on which the context launches its kernels."""
        s = ctypes.c_void_p()
        _check(load().psdns_gpu_get_stream(self._ctx, ctypes.byref(s)), "get_stream")
        return s.value or 0

    def profile(self, enable=True):
        _check(load().psdns_gpu_profile(self._ctx, 1 if enable else 0), "profile")

    def kernel_times(self):
        ms = np.zeros(6, np.float64)
        cnt = np.zeros(6, np.int64)
        _check(load().psdns_gpu_kernel_times(self._ctx, _dp(ms), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
               "kernel_times")
        return ms, cnt

    def particles_set(self, pos):
        """pos: (np, 3) FP64 positions in grid units (pp(np,1:3))."""
        a = np.asfortranarray(np.asarray(pos, np.float64))
        flat = np.ascontiguousarray(a.T)   # (3, np): column-major (np,3)
        self._np = flat.shape[1]
        _check(load().psdns_gpu_particles_set(self._ctx, self._np, _dp(flat)), "particles_set")

    def particles_init(self, nop, pstart=0, kipran=11):
        """partin.f positions, made at the next step's particle phase."""
        _check(load().psdns_gpu_particles_init(self._ctx, int(nop), int(pstart), int(kipran)), "particles_init")
        self._np = int(nop) if pstart == 0 else int(nop) ** 3

    def particles_advance(self, gsh1, dt_prev):
        """The particle phase of a step for drivers that call rk_stage themselves:
        before rk_stage(1), with that stage's shifts gsh(1:3,1) and the previous dt."""
        g = np.ascontiguousarray(gsh1, dtype=np.float64)
        _check(load().psdns_gpu_particles_advance(self._ctx, _dp(g), float(dt_prev)), "particles_advance")

    def particles_get(self):
        pos = np.zeros((3, self._np)); vel = np.zeros((3, self._np))
        _check(load().psdns_gpu_particles_get(self._ctx, _dp(pos), _dp(vel)), "particles_get")
        return pos.T.copy(), vel.T.copy()

    def spectra(self, which=FIELD_UN):
        """FP64 shell spectra (sptr.f): (ek[n], dk[n], eijk[n,6], stats dict)."""
        n = self.n
        ek = np.zeros(n); dk = np.zeros(n); e6 = np.zeros(n * 6); st = np.zeros(7)
        _check(load().psdns_gpu_spectra(self._ctx, int(which), _dp(ek), _dp(dk), _dp(e6), _dp(st)), "spectra")
        return ek, dk, e6.reshape(n, 6), dict(zip(["tke", "eps", "skew", "klen", "kvel", "ktime", "ekl"], st))

    def particles_write(self, prefix, ngp, istep, append=False):
        """pop1_write_local2.f output of one task (files under prefix/<igp>/)."""
        _check(load().psdns_gpu_particles_write(self._ctx, os.fsencode(prefix), int(ngp), int(istep),
                                                1 if append else 0), "particles_write")

    def write_checkpoint_set(self, prefix, iproc, jproc, which=FIELD_UN):
        """iproc*jproc pencil files <prefix>.p<t> (outpen_write_r.f layout)."""
        _check(load().psdns_gpu_write_checkpoint_set(self._ctx, os.fsencode(prefix), int(iproc), int(jproc),
                                                     int(which)), "write_checkpoint_set")

    def read_checkpoint_set(self, paths):
        arr = (ctypes.c_char_p * len(paths))(*[os.fsencode(p) for p in paths])
        _check(load().psdns_gpu_read_checkpoint_set(self._ctx, arr, len(paths)), "read_checkpoint_set")

    def write_chkptou(self, path, istep, iostep=1):
        _check(load().psdns_gpu_write_chkptou(self._ctx, os.fsencode(path), int(istep), int(iostep)), "write_chkptou")

    def read_chkptou(self, path, strict=True):
        """store.f icall 3; returns the stored istep."""
        ist = ctypes.c_int32()
        _check(load().psdns_gpu_read_chkptou(self._ctx, os.fsencode(path), 1 if strict else 0, ctypes.byref(ist)),
               "read_chkptou")
        return ist.value

    def write_ranout(self, path):
        _check(load().psdns_gpu_write_ranout(self._ctx, os.fsencode(path)), "write_ranout")

    def read_ranin(self, path):
        _check(load().psdns_gpu_read_ranin(self._ctx, os.fsencode(path)), "read_ranin")

    def filter_from(self, fine):
        """This (coarse) box's u and un := fine box's un inside this box's
        truncation sphere (psdns_gpu_filter_state)."""
        _check(load().psdns_gpu_filter_state(fine._ctx, self._ctx), "psdns_gpu_filter_state")

    def shell_factor(self, f):
        """Multiply the modes of shell i (1..len(f)-1) by f[i]."""
        f = np.ascontiguousarray(f, np.float64)
        _check(load().psdns_gpu_shell_factor(self._ctx, len(f) - 1, _dp(f)), "psdns_gpu_shell_factor")

    def corrector_features(self, which=FIELD_UN, nshell=None):
        k = resolved_shells(self.n) if nshell is None else int(nshell)
        x = np.zeros((k, CORRECTOR_FEATURES), np.float32)
        _check(load().psdns_gpu_corrector_features(self._ctx, int(which), k, _fp(x)), "corrector_features")
        return x

    def corrector_apply(self, corr):
        """Damp the resolved shells by the network's eddy viscosity over the
        last step's dt; returns (applied, max g)."""
        info = np.zeros(2)
        _check(load().psdns_gpu_corrector_apply(corr.handle, self._ctx, _dp(info)), "corrector_apply")
        return bool(info[0]), float(info[1])

    def write_checkpoint(self, path, which=FIELD_UN):
        """One-task pencil file in the reference's format (outpen_write_r.f)."""
        _check(load().psdns_gpu_write_checkpoint(self._ctx, os.fsencode(path), int(which)), "write_checkpoint")

    def read_checkpoint(self, path):
        _check(load().psdns_gpu_read_checkpoint(self._ctx, os.fsencode(path)), "read_checkpoint")

    def gradient_moments(self, which=FIELD_UN, gsh=(0.0, 0.0, 0.0)):
        """vgmomt.f: (moments 1..8 of du/dx, of dw/dz) on the grid shifted by gsh."""
        g = np.ascontiguousarray(gsh, dtype=np.float64)
        out = np.zeros(16, np.float64)
        _check(load().psdns_gpu_gradient_moments(self._ctx, int(which), _dp(g), _dp(out)), "gradient_moments")
        return out[:8].copy(), out[8:].copy()

    def transfer_spectrum(self, gsh=(0.0, 0.0, 0.0)):
        """trfsp.f: T(k), k = 1..n/2, on the grid shifted by gsh."""
        g = np.ascontiguousarray(gsh, dtype=np.float64)
        tk = np.zeros(self.n // 2)
        _check(load().psdns_gpu_transfer_spectrum(self._ctx, _dp(g), _dp(tk)), "transfer_spectrum")
        return tk

    def spectra_scales(self, which=FIELD_UN):
        """sptr.f one-dimensional spectra ([6, n/2+1] each) and scale statistics."""
        nh = self.n // 2 + 1
        xr = np.zeros(6 * nh); yr = np.zeros(6 * nh); zr = np.zeros(6 * nh); st = np.zeros(55)
        _check(load().psdns_gpu_spectra_scales(self._ctx, int(which), _dp(xr), _dp(yr), _dp(zr), _dp(st)),
               "spectra_scales")
        return xr.reshape(6, nh), yr.reshape(6, nh), zr.reshape(6, nh), {
            "corr": st[0:6], "lijk": st[6:24].reshape(6, 3), "rms": st[24:27], "raak": st[27:30],
            "ett": st[30:33], "tmij": st[33:42].reshape(3, 3), "grdiss": st[42],
            "taak": st[43:52].reshape(3, 3), "tmre": st[52:55]}

    def forcing_table(self):
        """for(kfor,k2fo,k2fo,3) of the last step as an array [3][k2fo][k2fo][kfor]."""
        kf = ctypes.c_int32()
        k2 = ctypes.c_int32()
        _check(load().psdns_gpu_forcing_table(self._ctx, None, ctypes.byref(kf), ctypes.byref(k2)), "forcing_table")
        tab = np.zeros(kf.value * k2.value * k2.value * 3, np.complex128)
        _check(load().psdns_gpu_forcing_table(self._ctx, _dp(tab.view(np.float64)), None, None), "forcing_table")
        return tab.reshape(3, k2.value, k2.value, kf.value)

    def forcing_stats(self):
        """Energy input of the last step (forcdt.f): efk per shell, eirate[3], erate."""
        kf = ctypes.c_int32()
        _check(load().psdns_gpu_forcing_table(self._ctx, None, ctypes.byref(kf), None), "forcing_table")
        efk = np.zeros(kf.value, np.float64)
        eir = np.zeros(3, np.float64)
        er = np.zeros(1, np.float64)
        _check(load().psdns_gpu_forcing_stats(self._ctx, _dp(efk), _dp(eir), _dp(er)), "forcing_stats")
        return {"efk": efk, "eirate": eir, "erate": er[0]}

    def time_info(self):
        out = np.zeros(4, np.float64)
        _check(load().psdns_gpu_get_time(self._ctx, _dp(out)), "get_time")
        return {"time": out[0], "dt": out[1], "velmax": out[2], "jstep": int(out[3])}


class Ensemble:
    """Independent boxes advanced together (psdns_gpu_ensemble_*): boxes of
    the same n share every kernel launch; fixed-dt boxes replay CUDA graphs."""

    def __init__(self, params_list):
        L = load()
        self.params = list(params_list)
        arr = (Params * len(self.params))(*self.params)
        self._ens = ctypes.c_void_p()
        _check(L.psdns_gpu_ensemble_create(arr, len(self.params), ctypes.byref(self._ens)),
               "psdns_gpu_ensemble_create")
        self.count = len(self.params)
        self.shapes = []
        for p in self.params:
            g = geometry(p.nx)
            self.shapes.append((3, g["xz_tot"], p.nx))

    def close(self):
        if self._ens:
            load().psdns_gpu_ensemble_destroy(self._ens)
            self._ens = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field_init(self, seeds):
        s = np.ascontiguousarray(seeds, dtype=np.int32)
        _check(load().psdns_gpu_ensemble_field_init(self._ens, s.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
               "ensemble_field_init")

    def set_state(self, box, un):
        a = np.ascontiguousarray(un, dtype=np.complex128)
        if a.shape != self.shapes[box]:
            raise ValueError(f"state shape {a.shape} != {self.shapes[box]}")
        _check(load().psdns_gpu_ensemble_set_state(self._ens, int(box), _dp(a.view(np.float64)), LAYOUT_YCYL),
               "ensemble_set_state")

    def get_state(self, box, which=FIELD_UN):
        out = np.zeros(self.shapes[box], np.complex128)
        _check(load().psdns_gpu_ensemble_get_state(self._ens, int(box), _dp(out.view(np.float64)), int(which),
                                                   LAYOUT_YCYL), "ensemble_get_state")
        return out

    def step(self, nsteps=1):
        """Advance every box nsteps steps; returns (status, info[count, 8])."""
        info = np.zeros((self.count, 8), np.float64)
        rc = load().psdns_gpu_ensemble_step(self._ens, int(nsteps), _dp(info))
        if rc not in (0, 2):
            _check(rc, "psdns_gpu_ensemble_step")
        return rc, info

    def tuning(self):
        """The autotuner's choice per class (psdns_gpu_ensemble_tuning)."""
        nc = ctypes.c_int32()
        _check(load().psdns_gpu_ensemble_tuning(self._ens, 0, None, ctypes.byref(nc)), "ensemble_tuning")
        out = np.zeros(8 * max(1, nc.value))
        _check(load().psdns_gpu_ensemble_tuning(self._ens, nc.value, _dp(out), ctypes.byref(nc)), "ensemble_tuning")
        keys = ("n", "boxes", "tuned", "boxes_per_launch", "k2_lines_per_block", "k4_lines_per_block",
                "default_ms", "chosen_ms")
        return [dict(zip(keys, [int(v) if j < 6 else float(v) for j, v in enumerate(out[8 * c:8 * c + 8])]))
                for c in range(nc.value)]

    def spectra(self, box, which=FIELD_UN):
        n = self.params[box].nx
        ek = np.zeros(n); dk = np.zeros(n); e6 = np.zeros(n * 6); st = np.zeros(7)
        _check(load().psdns_gpu_ensemble_spectra(self._ens, int(box), int(which), _dp(ek), _dp(dk), _dp(e6),
                                                 _dp(st)), "ensemble_spectra")
        return ek, dk, e6.reshape(n, 6), dict(zip(["tke", "eps", "skew", "klen", "kvel", "ktime", "ekl"], st))
