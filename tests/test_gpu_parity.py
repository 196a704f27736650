"""GPU parity: the sm_100a RK2 step against the FP64 oracle, through the
C-ABI (psdns_gpu.Solver).

Tolerances (relative L2 over the whole state, and per E(k) shell):
  FP64 device state: 1e-11 (both sides are FP64; differences are FFT
                     rounding order only)
  FP32 device state: 2e-5 after 5 steps (FP32 FFTs, ~1e-7 per operation)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def shell_spectrum(un, geo, n):
    """E(k) per shell, ik = int(k + 1.5) (sptr.f:161-165), kx=0 plane once."""
    col = geo["colstart"]
    kk = lambda i: np.where(i > n // 2, i - n, i)
    ky = kk(np.arange(n))
    E = np.zeros(n)
    for x in range(len(col) - 1):
        tf = 1.0 if x == 0 else 2.0
        for a in range(col[x], col[x + 1]):
            z = geo["az"][a]
            k = np.sqrt(x * x + ky ** 2 + kk(z) ** 2)
            ik = (k + 1.5).astype(int)
            e = 0.5 * tf * np.sum(np.abs(un[:, a, :]) ** 2, axis=0)
            np.add.at(E, ik, e)
    return E


def run_pair(oracle_mod, gpu_mod, n, prec, steps, kshift=1, cfl=-1.0, dt=0.005, nu=0.01, seed=1234):
    o = oracle_mod.Oracle(n, nu, cfl=cfl, dt=dt, kshift=kshift)
    un0 = o.field_init(seed)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=cfl, dt=dt, kshift=kshift,
                       seed_input=o_seed_default())
    s.set_state(un0)
    infos = []
    for _ in range(steps):
        assert o.step() == 0
        info = s.step()
        assert info["status"] == 0
        infos.append((o.scalars(), info))
    u_o, un_o = o.get_state()
    u_g = s.get_state(gpu_mod.FIELD_U)
    un_g = s.get_state(gpu_mod.FIELD_UN)
    geo = o.geometry()
    o.close()
    s.close()
    return u_o, un_o, u_g, un_g, infos, geo


def o_seed_default():
    return 122929298


@pytest.mark.parametrize("n", [16, 32, 48, 64, 96])
def test_fp64_one_step(oracle_mod, gpu_mod, n):
    u_o, un_o, u_g, un_g, infos, geo = run_pair(oracle_mod, gpu_mod, n, gpu_mod.PREC_FP64, 1)
    so, sg = infos[0]
    np.testing.assert_array_equal(sg["gsh1"], so["gsh"][:, 0])
    assert abs(sg["velmax"] - so["velmax"]) <= 1e-12 * so["velmax"]
    assert rel_l2(un_g, un_o) < 1e-11
    assert rel_l2(u_g, u_o) < 1e-11


def test_fp64_five_steps_adaptive_dt(oracle_mod, gpu_mod):
    n = 32
    u_o, un_o, u_g, un_g, infos, geo = run_pair(oracle_mod, gpu_mod, n, gpu_mod.PREC_FP64, 5, cfl=1.0)
    for so, sg in infos:
        assert abs(sg["dt"] - so["dt"]) <= 1e-12 * so["dt"]
    assert rel_l2(un_g, un_o) < 1e-11
    Eo, Eg = shell_spectrum(un_o, geo, n), shell_spectrum(un_g, geo, n)
    m = Eo > 1e-30
    assert np.max(np.abs(Eg[m] - Eo[m]) / Eo[m]) < 1e-10


@pytest.mark.parametrize("n", [32, 48, 64])
def test_fp32_five_steps(oracle_mod, gpu_mod, n):
    u_o, un_o, u_g, un_g, infos, geo = run_pair(oracle_mod, gpu_mod, n, gpu_mod.PREC_FP32, 5)
    err = rel_l2(un_g, un_o)
    assert err < 2e-5, err
    Eo, Eg = shell_spectrum(un_o, geo, n), shell_spectrum(un_g, geo, n)
    m = Eo > 1e-8 * Eo.max()
    assert np.max(np.abs(Eg[m] - Eo[m]) / Eo[m]) < 1e-4


@pytest.mark.parametrize("kshift", [2, 3, 4])
def test_shift_modes(oracle_mod, gpu_mod, kshift):
    u_o, un_o, u_g, un_g, infos, geo = run_pair(oracle_mod, gpu_mod, 32, gpu_mod.PREC_FP64, 2, kshift=kshift)
    assert rel_l2(un_g, un_o) < 1e-11


def test_rk_stage_entry_point(oracle_mod, gpu_mod):
    """psdns_gpu_rk_stage with driver-supplied shifts and dt."""
    n = 32
    o = oracle_mod.Oracle(n, 0.01, cfl=-1, dt=0.004, kshift=4)
    un0 = o.field_init(99)
    o.set_state(un0)
    gsh = np.array([[0.1, 0.6], [0.3, 0.8], [0.45, 0.95]])
    o.set_shifts(gsh)
    o.stage(1)
    o.stage(2)
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=0.01, cfl=-1, dt=0.004, kshift=4)
    s.set_state(un0)
    vm = s.rk_stage(1, gsh, dt=0.004)
    s.rk_stage(2, gsh)
    assert abs(vm - o.scalars()["velmax"]) < 1e-12 * vm
    _, un_o = o.get_state()
    assert rel_l2(s.get_state(gpu_mod.FIELD_UN), un_o) < 1e-11
    o.close(); s.close()


@pytest.mark.parametrize("prec,tol", [(1, 1e-13), (0, 1e-6)])
def test_device_field_init_matches_oracle(oracle_mod, gpu_mod, prec, tol):
    """field.f restated on the device (jump-ahead LCG) against the sequential oracle."""
    n = 32
    o = oracle_mod.Oracle(n, 0.01, kshift=4)
    ref = o.field_init(2024)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=-1, dt=0.005, kshift=4)
    s.field_init(2024)
    got = s.get_state(gpu_mod.FIELD_UN)
    assert rel_l2(got, ref) < tol
    np.testing.assert_array_equal(s.get_state(gpu_mod.FIELD_U), got)
    o.close(); s.close()


@pytest.mark.parametrize("tfiuo,cfl", [(0.0, -1.0), (0.4, -1.0), (0.0, np.pi), (0.4, np.pi)])
def test_forced_steps_match_oracle(oracle_mod, gpu_mod, tfiuo, cfl):
    """Eswaran-Pope forcing (force.f with vfuo.f, or vfiuo.f + raniuo.f), FP64
    device state.  With a fixed dt the forcing table depends only on the RNG
    path and must be bit-identical; with adaptive dt (cfl = pi, Courant number
    0.5) it also depends on dt = cfl/velmax, whose device value differs from
    the oracle's in the last bits, so the table is compared to 1e-11."""
    n, nu = 32, 0.02
    kforce, tforce = 2.99, 0.5
    epsfor = 0.1 / (4.0 * (4.0 * np.pi / 3.0) * kforce ** 3)
    dt = 0.004 if cfl < 0 else 0.0
    o = oracle_mod.Oracle(n, nu, cfl=cfl, dt=dt, kshift=1)
    o.set_forcing(kforce, tforce, epsfor, tfiuo)
    un0 = o.field_init(77)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=nu, cfl=cfl, dt=dt, kshift=1,
                       kforce=kforce, tforce=tforce, epsfor=epsfor, tfiuo=tfiuo)
    s.set_state(un0)
    for step in range(3):
        o.step()
        info = s.step()
        so = o.scalars()
        assert abs(info["dt"] - so["dt"]) <= 1e-12 * so["dt"]
        tab_o, ef_o = o.forcing()
        tab_g = s.forcing_table()
        if cfl < 0:
            np.testing.assert_array_equal(tab_g, tab_o)
        else:
            np.testing.assert_allclose(tab_g, tab_o, rtol=1e-11, atol=1e-11 * np.abs(tab_o).max())
        st = s.forcing_stats()
        efk_o = 0.5 * ef_o.sum(axis=1) / so["dt"]
        np.testing.assert_allclose(st["efk"], efk_o, rtol=1e-9, atol=1e-15)
    _, un_o = o.get_state()
    assert rel_l2(s.get_state(gpu_mod.FIELD_UN), un_o) < 1e-11
    o.close(); s.close()


@pytest.mark.parametrize("prec,tol", [(1, 1e-12), (0, 1e-5)])
def test_spectra_match_oracle(oracle_mod, gpu_mod, prec, tol):
    """FP64 shell sums on the device (sptr.f) against the oracle after 2 steps."""
    n, nu = 32, 0.01
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=0.005, kshift=1)
    un0 = o.field_init(5)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=-1, dt=0.005, kshift=1)
    s.set_state(un0)
    for _ in range(2):
        o.step()
        s.step()
    ek_o, dk_o, e6_o, st_o = o.spectra(1)
    ek_g, dk_g, e6_g, st_g = s.spectra(gpu_mod.FIELD_UN)
    # FP32 state: shells holding >= 1e-6 of the peak agree to 1e-5; the
    # near-empty tail shells (down to 1e-10 of the peak) to 1e-4
    m = ek_o > 1e-6 * ek_o.max()
    np.testing.assert_allclose(ek_g[m], ek_o[m], rtol=tol)
    np.testing.assert_allclose(dk_g[m], dk_o[m], rtol=tol)
    m = ek_o > 1e-10 * ek_o.max()
    np.testing.assert_allclose(ek_g[m], ek_o[m], rtol=1e-4 if prec == 0 else tol)
    for k in ("tke", "eps", "skew", "klen", "ekl"):
        assert abs(st_g[k] - st_o[k]) <= tol * abs(st_o[k]), k
    o.close(); s.close()


@pytest.mark.parametrize("prec,tol_p,tol_v", [(1, 1e-11, 1e-9), (0, 1e-6, 2e-4)])
def test_particles_match_oracle(oracle_mod, gpu_mod, prec, tol_p, tol_v):
    """Particles: spectral-prefilter spline + warp-cooperative interpolation on
    the device against the oracle's tridiagonal spline sweeps
    (spxyz_m.f/solsp1.f) and spcal_local.f interpolation; 4 steps, random
    shifts, FP64 positions."""
    n, nu = 32, 0.01
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=0.01, kshift=1)
    un0 = o.field_init(9)
    o.set_state(un0)
    rng = np.random.default_rng(3)
    pos = 1.0 + rng.random((500, 3)) * n
    o.particles_set(pos)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=-1, dt=0.01, kshift=1)
    s.set_state(un0)
    s.particles_set(pos)
    for _ in range(4):
        o.step()
        s.step()
    po, vo = o.particles_get()
    pg, vg = s.particles_get()
    assert np.abs(pg - po).max() < tol_p * n
    assert np.abs(vg - vo).max() < tol_v * np.abs(vo).max()
    assert np.abs(pg - pos).max() > 0.05     # they did move
    o.close(); s.close()


@pytest.mark.parametrize("prec,tol_p,tol_v", [(1, 1e-11, 1e-9), (0, 1e-6, 2e-4)])
def test_particles_edge_positions(oracle_mod, gpu_mod, prec, tol_p, tol_v):
    """Positions the cell search must fold: far outside the box on both sides
    (partsp.f keeps unwrapped coordinates; spcal_local.f folds ipx mod n with
    a 1000 n offset for negatives), exactly on grid planes, and on the
    periodic seam."""
    n, nu = 32, 0.01
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=0.01, kshift=1)
    un0 = o.field_init(11)
    o.set_state(un0)
    rng = np.random.default_rng(8)
    far = rng.uniform(-3 * n, 4 * n, size=(200, 3))
    planes = rng.integers(-2 * n, 3 * n, size=(100, 3)).astype(np.float64)
    seam = np.array([[0.0, 1.0, float(n)], [float(n + 1), 1.0 - 1e-12, 0.5], [1.0, 1.0, 1.0],
                     [-1.0, -float(n), 2.0 * n + 1.0]])
    pos = np.concatenate([far, planes, seam])
    o.particles_set(pos)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=nu, cfl=-1, dt=0.01, kshift=1)
    s.set_state(un0)
    s.particles_set(pos)
    for _ in range(3):
        o.step()
        s.step()
    po, vo = o.particles_get()
    pg, vg = s.particles_get()
    assert np.abs(pg - po).max() < tol_p * n
    assert np.abs(vg - vo).max() < tol_v * np.abs(vo).max()
    o.close(); s.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_particles_advance_with_rk_stage(gpu_mod, prec):
    """A driver that runs the stages itself (rk_stage with its own shifts and
    dt) and calls particles_advance before stage 1 moves the particles exactly
    as psdns_gpu_step does (zero shifts, kshift = 4, so both paths use the
    same grid)."""
    n, nu, dt = 32, 0.01, 0.01
    kw = dict(n=n, precision=prec, viscos=nu, cfl=-1, dt=dt, kshift=4, kforce=0.0)
    a = gpu_mod.Solver(**kw)
    b = gpu_mod.Solver(**kw)
    a.field_init(5)
    b.set_state(a.get_state(gpu_mod.FIELD_UN))
    pos = 1.0 + np.random.default_rng(4).random((300, 3)) * n
    a.particles_set(pos)
    b.particles_set(pos)
    gsh = np.zeros((3, 2))
    dt_prev = 0.0
    for _ in range(3):
        assert a.step()["status"] == 0
        b.particles_advance(gsh[:, 0], dt_prev)
        b.rk_stage(1, gsh, dt)
        b.rk_stage(2, gsh)
        dt_prev = dt
    pa, va = a.particles_get()
    pb, vb = b.particles_get()
    np.testing.assert_array_equal(pb, pa)
    np.testing.assert_array_equal(vb, va)
    np.testing.assert_array_equal(b.get_state(gpu_mod.FIELD_UN), a.get_state(gpu_mod.FIELD_UN))
    assert np.abs(pa - pos).max() > 0.05
    a.close(); b.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_full_layout_round_trip(oracle_mod, gpu_mod, prec):
    """PSDNS_LAYOUT_FULL: u(nxh,ny,nz,nv) <-> cylinder columns (x, ., z)."""
    n = 32
    o = oracle_mod.Oracle(n, 0.01)
    un = o.field_init(55)
    geo = o.geometry()
    o.close()
    s = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=-1.0, dt=0.005)
    s.set_state(un)
    full = s.get_state(gpu_mod.FIELD_UN, layout=gpu_mod.LAYOUT_FULL)
    assert full.shape == (3, n, n, n // 2 + 1)
    kx = np.repeat(np.arange(len(geo["colstart"]) - 1), np.diff(geo["colstart"]))
    expect = np.zeros_like(full)
    expect[:, geo["az"], :, kx] = un.transpose(1, 0, 2)
    tol = 0 if prec == 1 else 1e-6
    np.testing.assert_allclose(full, expect, rtol=0, atol=tol * np.abs(un).max())
    # back through the full layout: the cylinder is reproduced
    s2 = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=-1.0, dt=0.005)
    s2.set_state(full, layout=gpu_mod.LAYOUT_FULL)
    np.testing.assert_allclose(s2.get_state(gpu_mod.FIELD_UN), s.get_state(gpu_mod.FIELD_UN), rtol=0, atol=0)
    s.close()
    s2.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_async_state_copies_match_sync(oracle_mod, gpu_mod, prec):
    """set_state_async / step / get_state_async into the same pinned host
    buffer, three times, then sync: equal to the synchronous calls."""
    import torch
    n = 32
    o = oracle_mod.Oracle(n, 0.01)
    un0 = o.field_init(21)
    o.close()
    a = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=1.0)
    b = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=1.0)
    nbytes = un0.size * 16
    host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    view = host.numpy().view(np.complex128).reshape(un0.shape)
    view[...] = un0
    for _ in range(3):
        a.set_state_async_ptr(host.data_ptr())
        a.step()
        a.get_state_async_ptr(host.data_ptr())
    a.sync()
    b.set_state(un0)
    cur = un0
    for _ in range(3):
        b.set_state(cur)
        b.step()
        cur = b.get_state()
    np.testing.assert_array_equal(view, cur)
    a.close()
    b.close()


@pytest.mark.parametrize("prec,tol", [(1, 1e-10), (0, 1e-4)])
def test_gradient_moments_match_oracle(oracle_mod, gpu_mod, prec, tol):
    """vgmomt.f moments of du/dx and dw/dz, shifted grid, after two steps."""
    n = 32
    o = oracle_mod.Oracle(n, 0.01, cfl=1.0, kshift=1)
    un0 = o.field_init(8)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=1.0, kshift=1)
    s.set_state(un0)
    for _ in range(2):
        o.step()
        s.step()
    gsh = (0.3, 0.71, 0.05)
    for which in (gpu_mod.FIELD_U, gpu_mod.FIELD_UN):
        mo = o.gradient_moments(which, gsh)
        mg = s.gradient_moments(which, gsh)
        for f in range(2):
            # even moments relative; odd ones against the scale of the even ones
            for m in range(8):
                scale = mo[f][m] if m % 2 == 1 else mo[f][1] ** ((m + 1) / 2)
                assert abs(mg[f][m] - mo[f][m]) <= tol * abs(scale), (which, f, m, mg[f][m], mo[f][m])
    # the diagnostic leaves the run untouched
    o.step()
    s.step()
    _, un_o = o.get_state()
    assert rel_l2(s.get_state(gpu_mod.FIELD_UN), un_o) < (1e-11 if prec == 1 else 2e-5)
    o.close()
    s.close()


def _read_pencil_file(path, n, nv):
    """Independent reader of the single-task outpen_write_r.f layout:
    big-endian records with 4-byte markers; per variable (i,nx,ny,nz),
    (xist,xisz,zjst,zjsz,1,ny), then two records per z (not Nyquist)."""
    import struct
    raw = open(path, "rb").read()
    pos = 0
    recs = []
    while pos < len(raw):
        (ln,) = struct.unpack(">i", raw[pos:pos + 4])
        recs.append(raw[pos + 4:pos + 4 + ln])
        (ln2,) = struct.unpack(">i", raw[pos + 4 + ln:pos + 8 + ln])
        assert ln2 == ln
        pos += 8 + ln
    out = np.zeros((nv, n, n, n // 2), complex)    # [v][z][y][kx < n/2]
    r = 0
    for v in range(nv):
        assert struct.unpack(">4i", recs[r]) == (v + 1, n, n, n)
        assert struct.unpack(">6i", recs[r + 1]) == (1, n // 2, 1, n, 1, n)
        r += 2
        for z in range(n):
            if z == n // 2:
                continue
            for ys in (range(0, n // 2), range(n // 2 + 1, n)):
                a = np.frombuffer(recs[r], dtype=">f8").reshape(len(ys), n // 2, 2)
                out[v, z, ys.start:ys.stop, :] = a[..., 0] + 1j * a[..., 1]
                r += 1
    assert r == len(recs)
    return out


@pytest.mark.parametrize("nc", [0, 1])
def test_checkpoint_files_in_reference_format(tmp_path, oracle_mod, gpu_mod, nc):
    n = 32
    o = oracle_mod.Oracle(n, 0.01)
    un0 = o.field_init(5)
    o.close()
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=0.01, cfl=1.0, nc=nc, pr=0.7, grad=(0, 1, 0))
    st = np.zeros(s.state_shape(), complex)
    st[:3] = un0
    if nc:
        st[3] = un0[0] * 0.3
    s.set_state(st)
    s.step()
    path = str(tmp_path / "outpenc.p0")
    s.write_checkpoint(path)
    got = _read_pencil_file(path, n, 3 + nc)
    full = s.get_state(gpu_mod.FIELD_UN, layout=gpu_mod.LAYOUT_FULL)
    expect = full[..., : n // 2].copy()
    expect[:, n // 2, :, :] = 0
    expect[:, :, n // 2, :] = 0
    np.testing.assert_array_equal(got, expect)
    s2 = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=0.01, cfl=1.0, nc=nc, pr=0.7, grad=(0, 1, 0))
    s2.read_checkpoint(path)
    np.testing.assert_array_equal(s2.get_state(gpu_mod.FIELD_UN), s.get_state(gpu_mod.FIELD_UN))
    s.close()
    s2.close()


@pytest.mark.parametrize("pstart,nop", [(0, 500), (-1, 4)])
def test_partin_matches_oracle(oracle_mod, gpu_mod, pstart, nop):
    """partin.f positions from the kipran RNG sequence (bit-exact: host
    arithmetic on both sides), then 3 particle steps (FP64 device)."""
    n, nu = 32, 0.01
    o = oracle_mod.Oracle(n, nu, cfl=-1, dt=0.01, kshift=1)
    un0 = o.field_init(9)
    o.set_state(un0)
    o.particles_init(nop, pstart, 11)
    s = gpu_mod.Solver(n=n, precision=gpu_mod.PREC_FP64, viscos=nu, cfl=-1, dt=0.01, kshift=1)
    s.set_state(un0)
    s.particles_init(nop, pstart, 11)
    o.step()
    s.step()
    po, vo = o.particles_get()
    pg, vg = s.particles_get()
    np.testing.assert_array_equal(pg, po)
    assert np.abs(vg - vo).max() < 1e-9 * np.abs(vo).max()
    for _ in range(2):
        o.step()
        s.step()
    po, _ = o.particles_get()
    pg, _ = s.particles_get()
    assert np.abs(pg - po).max() < 1e-11 * n
    o.close()
    s.close()


@pytest.mark.parametrize("prec,tol", [(1, 1e-11), (0, 1e-5)])
def test_spectra_scales_match_oracle(oracle_mod, gpu_mod, prec, tol):
    """sptr.f one-dimensional spectra and scales after two steps."""
    n = 32
    o = oracle_mod.Oracle(n, 0.01, cfl=1.0, kshift=1)
    un0 = o.field_init(71)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=1.0, kshift=1)
    s.set_state(un0)
    for _ in range(2):
        o.step()
        s.step()
    for which in (gpu_mod.FIELD_U, gpu_mod.FIELD_UN):
        xo, yo, zo, so = o.spectra_scales(which)
        xg, yg, zg, sg = s.spectra_scales(which)
        for a, b in ((xg, xo), (yg, yo), (zg, zo)):
            m = np.abs(b) > 1e-6 * np.abs(b).max()
            assert np.max(np.abs(a[m] - b[m]) / np.abs(b[m])) < tol
        for k in so:
            np.testing.assert_allclose(sg[k], so[k], rtol=tol, atol=tol * np.abs(so[k]).max() * 1e-3)
    o.close()
    s.close()


@pytest.mark.parametrize("prec,tol", [(1, 1e-10), (0, 1e-4)])
def test_transfer_spectrum_matches_oracle(oracle_mod, gpu_mod, prec, tol):
    """trfsp.f transfer spectrum after one step, shifted grid; the state is
    unchanged by the diagnostic."""
    n = 32
    o = oracle_mod.Oracle(n, 0.01, cfl=1.0, kshift=1)
    un0 = o.field_init(13)
    o.set_state(un0)
    s = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=1.0, kshift=1)
    s.set_state(un0)
    o.step()
    s.step()
    gsh = (0.25, 0.5, 0.8)
    to = o.transfer_spectrum(gsh)
    tg = s.transfer_spectrum(gsh)
    scale = np.abs(to).max()
    assert np.abs(tg - to).max() < tol * scale
    o.step()
    s.step()
    _, un_o = o.get_state()
    assert rel_l2(s.get_state(gpu_mod.FIELD_UN), un_o) < (1e-11 if prec == 1 else 2e-5)
    o.close()
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,nc", [(0, 0), (1, 0), (0, 1)])
def test_sphere_copies(gpu_mod, oracle_mod, prec, nc):
    """psdns_gpu_{set,get}_state_sphere_async: the entries inside the
    truncation sphere (masks.f) move between pinned host memory and the
    device; the others are neither read nor written.  A stepping loop that
    downloads and re-uploads through the same pinned array matches the
    synchronous path."""
    import torch
    n = 32
    kw = dict(nc=1, pr=1.0, grad=(0.0, 1.0, 0.0)) if nc else {}
    s = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=-1.0, dt=0.005, kshift=1, **kw)
    s.field_init(7)
    ref = s.get_state(gpu_mod.FIELD_UN)
    if nc:   # give the scalar a field of its own (stored in the device precision)
        ref[3] = 0.1 * ref[0]
        s.set_state(ref)
        ref = s.get_state(gpu_mod.FIELD_UN)
    o = oracle_mod.Oracle(n, 0.01, kshift=4)
    kym = o.geometry()["kymax"].astype(np.int64)
    o.close()
    np.testing.assert_array_equal(gpu_mod.geometry(n)["kymax"], kym)
    y = np.arange(n)
    ky = np.minimum(y, n - y)
    inside = (y[None, :] != n // 2) & (ky[None, :] <= kym[:, None])       # [xz_tot, n]
    np.testing.assert_array_equal(gpu_mod.sphere_mask(n), inside)
    shape = s.state_shape()
    host = torch.empty(int(np.prod(shape)) * 2, dtype=torch.float64, pin_memory=True)
    h = host.numpy().view(np.complex128).reshape(shape)
    h[...] = 7.0 + 3.0j                                                       # sentinel
    s.get_state_sphere_async_ptr(host.data_ptr())
    s.sync()
    np.testing.assert_array_equal(h[:, inside], ref[:, inside])
    assert np.all(h[:, ~inside] == 7.0 + 3.0j)
    # upload a modified field through the sphere path; outside entries of the
    # host array are ignored
    h[:, inside] *= 0.5
    h[:, ~inside] = 1e30
    s.set_state_sphere_async_ptr(host.data_ptr())
    s.sync()
    got = s.get_state(gpu_mod.FIELD_UN)
    np.testing.assert_allclose(got[:, inside], 0.5 * ref[:, inside], rtol=1e-6 if prec == 0 else 0)
    # stepping loop through the same array == synchronous stepping
    t = gpu_mod.Solver(n=n, precision=prec, viscos=0.01, cfl=-1.0, dt=0.005, kshift=1, **kw)
    t.set_state(got)
    h[...] = 0
    h[:, inside] = got[:, inside]
    for _ in range(3):
        s.set_state_sphere_async_ptr(host.data_ptr())
        s.step()
        s.get_state_sphere_async_ptr(host.data_ptr())
        t.step()
    s.sync()
    want = t.get_state(gpu_mod.FIELD_UN)
    np.testing.assert_array_equal(h[:, inside], want[:, inside])
    s.close()
    t.close()


def test_error_paths_leave_context_usable(gpu_mod):
    """Refused calls return an error status with a message and change
    nothing: sphere copies from pageable memory, a particle step without
    particles, a stage-1 call without dt."""
    n = 32
    s = gpu_mod.Solver(n=n, precision=0, viscos=0.01, cfl=-1.0, dt=0.005, kshift=1)
    s.field_init(3)
    before = s.get_state(gpu_mod.FIELD_UN)
    pageable = np.zeros(int(np.prod(s.state_shape())) * 2)
    with pytest.raises(RuntimeError, match="pinned"):
        s.set_state_sphere_async_ptr(pageable.ctypes.data)
    with pytest.raises(RuntimeError, match="pinned"):
        s.get_state_sphere_async_ptr(pageable.ctypes.data)
    with pytest.raises(RuntimeError, match="no particles"):
        s.particles_advance(np.zeros(3), 0.005)
    with pytest.raises(RuntimeError, match="dt"):
        s.rk_stage(1, np.zeros((3, 2)), dt=0.0)
    s.sync()
    np.testing.assert_array_equal(s.get_state(gpu_mod.FIELD_UN), before)
    assert s.step()["status"] == 0
    s.close()


def test_sphere_download_then_step_keeps_the_old_state(gpu_mod):
    """A step issued right after a sphere download must not overwrite the
    state while the download still reads it: the host array holds the
    state before the step, and an upload issued later is ordered after it."""
    import torch
    n = 32
    s = gpu_mod.Solver(n=n, precision=1, viscos=0.01, cfl=-1.0, dt=0.005, kshift=1)
    s.field_init(21)
    before = s.get_state(gpu_mod.FIELD_UN)
    inside = gpu_mod.sphere_mask(n)
    shape = s.state_shape()
    host = torch.zeros(int(np.prod(shape)) * 2, dtype=torch.float64, pin_memory=True)
    h = host.numpy().view(np.complex128).reshape(shape)
    for _ in range(3):
        s.get_state_sphere_async_ptr(host.data_ptr())
        s.step()
    s.sync()
    after = s.get_state(gpu_mod.FIELD_UN)
    # the last download read the state of the step before the last one
    s2 = gpu_mod.Solver(n=n, precision=1, viscos=0.01, cfl=-1.0, dt=0.005, kshift=1)
    s2.set_state(before)
    s2.step()
    s2.step()
    want = s2.get_state(gpu_mod.FIELD_UN)
    np.testing.assert_array_equal(h[:, inside], want[:, inside])
    assert not np.array_equal(want[:, inside], after[:, inside])
    s.close(); s2.close()


def test_host_register_for_sphere_copies(gpu_mod):
    """psdns_gpu_host_register pins an ordinary host array in place (what a
    Fortran driver would do with its uy array) so that the sphere copies can
    use it; after psdns_gpu_host_unregister they refuse it again."""
    n = 32
    s = gpu_mod.Solver(n=n, precision=1, viscos=0.01, cfl=-1.0, dt=0.005, kshift=1)
    s.field_init(2)
    ref = s.get_state(gpu_mod.FIELD_UN)
    inside = gpu_mod.sphere_mask(n)
    h = np.zeros(s.state_shape(), np.complex128)
    gpu_mod.host_register(h)
    try:
        s.get_state_sphere_async_ptr(h.ctypes.data)
        s.sync()
        np.testing.assert_array_equal(h[:, inside], ref[:, inside])
        h[:, inside] *= 2.0
        s.set_state_sphere_async_ptr(h.ctypes.data)
        s.sync()
        np.testing.assert_array_equal(s.get_state(gpu_mod.FIELD_UN)[:, inside], 2.0 * ref[:, inside])
    finally:
        gpu_mod.host_unregister(h)
    with pytest.raises(RuntimeError, match="pinned"):
        s.get_state_sphere_async_ptr(h.ctypes.data)
    s.close()
