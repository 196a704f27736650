"""Restart from files in the reference's formats: a run interrupted after a
few steps writes its state as a multi-task pencil set
(homogeneous/outpen_write_r.f), its checkpoint metadata (store.f icall 2,
chkptou) and its RNG seeds (ranseq.f k = -2, ranout); a new context reads
them (inpen_read_r.f, store.f icall 3, ranseq.f k = -1) and continues.

* unforced, fixed dt, kshift 4: the continued run is bit-identical to the
  uninterrupted one;
* forced (vfuo.f and vfiuo.f processes), kshift 1: the RNG seed tables are
  identical after the same number of steps; the forcing processes, time and
  gsh(:,2) travel through the 9 significant digits of store.f's format 910,
  so the states agree to 1e-7 relative L2 (FP64) rather than bit for bit;
* a pencil set of 1 x 1 tasks is byte-identical to the one-task file, and a
  set whose pencils overlap or leave a gap is refused."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make(P, forced, tfiuo=0.0, kshift=1):
    kw = dict(n=32, precision=P.PREC_FP64, viscos=0.02, cfl=-1.0, dt=0.004, kshift=kshift)
    if forced:
        kw.update(kforce=2.99, tforce=0.5, epsfor=0.1 / (4.0 * (4.0 * np.pi / 3.0) * 2.99 ** 3), tfiuo=tfiuo)
    return P.Solver(**kw)


def run_and_restart(P, tmp_path, forced, tfiuo=0.0, kshift=1, before=3, after=3):
    a = make(P, forced, tfiuo, kshift)
    a.field_init(4242)
    for _ in range(before):
        a.step()
    prefix = str(tmp_path / "outpen")
    a.write_checkpoint_set(prefix, 2, 4)
    a.write_chkptou(str(tmp_path / "chkptou"), istep=before, iostep=5)
    a.write_ranout(str(tmp_path / "ranout"))
    for _ in range(after):
        a.step()
    b = make(P, forced, tfiuo, kshift)
    b.read_checkpoint_set([f"{prefix}.p{t}" for t in range(8)])
    assert b.read_chkptou(str(tmp_path / "chkptou"), strict=True) == before
    b.read_ranin(str(tmp_path / "ranout"))
    for _ in range(after):
        b.step()
    a.write_ranout(str(tmp_path / "ranout_a"))
    b.write_ranout(str(tmp_path / "ranout_b"))
    seeds_equal = open(tmp_path / "ranout_a").read() == open(tmp_path / "ranout_b").read()
    out = (a.get_state(P.FIELD_UN), b.get_state(P.FIELD_UN), seeds_equal)
    tab = (a.forcing_table(), b.forcing_table()) if forced else None
    a.close()
    b.close()
    return out, tab


def test_unforced_restart_is_bit_identical(gpu_mod, tmp_path):
    (ua, ub, seeds), _ = run_and_restart(gpu_mod, tmp_path, forced=False, kshift=4)
    assert seeds
    np.testing.assert_array_equal(ua, ub)


@pytest.mark.parametrize("tfiuo", [0.0, 0.4])
def test_forced_restart_continues_the_run(gpu_mod, tmp_path, tfiuo):
    (ua, ub, seeds), (ta, tb) = run_and_restart(gpu_mod, tmp_path, forced=True, tfiuo=tfiuo, kshift=1)
    assert seeds
    assert rel(ub, ua) < 1e-7
    np.testing.assert_allclose(tb, ta, rtol=0, atol=1e-7 * np.abs(ta).max())


def test_chkptou_records_and_strict_check(gpu_mod, tmp_path):
    P = gpu_mod
    a = make(P, True)
    a.field_init(1)
    a.step()
    path = str(tmp_path / "chkptou")
    a.write_chkptou(path, istep=1, iostep=5)
    lines = open(path).read().splitlines()
    assert [int(lines[0][8 * i:8 * i + 8]) for i in range(4)][:2] == [13, 18]   # nic2, nrc2 (nc = 0: ncd = 1)
    assert lines[1][:24] == "      32      32      32"
    # a run with another viscosity refuses the file under kstop = 1
    b = P.Solver(n=32, precision=P.PREC_FP64, viscos=0.03, cfl=-1.0, dt=0.004, kshift=1, kforce=2.99, tforce=0.5,
                 epsfor=0.1 / (4.0 * (4.0 * np.pi / 3.0) * 2.99 ** 3))
    with pytest.raises(P.PsdnsError, match="real no. 1"):
        b.read_chkptou(path, strict=True)
    b.read_chkptou(path, strict=False)
    a.close()
    b.close()


def test_pencil_sets(gpu_mod, tmp_path):
    P = gpu_mod
    a = make(P, False)
    a.field_init(9)
    a.step()
    a.write_checkpoint(str(tmp_path / "one"))
    a.write_checkpoint_set(str(tmp_path / "set"), 1, 1)
    assert open(tmp_path / "one", "rb").read() == open(tmp_path / "set.p0", "rb").read()
    a.write_checkpoint_set(str(tmp_path / "four"), 4, 1)
    b = make(P, False)
    with pytest.raises(P.PsdnsError, match="does not cover"):
        b.read_checkpoint_set([str(tmp_path / f"four.p{t}") for t in range(3)])
    with pytest.raises(P.PsdnsError, match="given twice"):
        b.read_checkpoint_set([str(tmp_path / f"four.p{t}") for t in (0, 1, 2, 3, 3)])
    b.read_checkpoint_set([str(tmp_path / f"four.p{t}") for t in (3, 1, 0, 2)])
    np.testing.assert_array_equal(b.get_state(P.FIELD_UN), a.get_state(P.FIELD_UN))
    a.close()
    b.close()


def _records(path):
    """Fortran sequential unformatted, big-endian 4-byte record markers
    (an independent reader of the reference's particle files)."""
    import struct
    data = open(path, "rb").read()
    out, o = [], 0
    while o < len(data):
        (m,) = struct.unpack(">i", data[o:o + 4])
        out.append(data[o + 4:o + 4 + m])
        (m2,) = struct.unpack(">i", data[o + 4 + m:o + 8 + m])
        assert m2 == m
        o += 8 + m
    return out


def test_particle_output_in_the_reference_layout(gpu_mod, tmp_path):
    """psdns_gpu_particles_get's pp(np, 1:6) order through the writer of
    pop1_write_local2.f (two groups of tetrads) and back."""
    import struct
    P = gpu_mod
    ngp, nrefp = 2, 300
    np_ = nrefp * (1 + 3 * ngp)
    s = make(P, False)
    s.field_init(3)
    rng = np.random.default_rng(8)
    s.particles_set(1.0 + rng.random((np_, 3)) * 32)
    for g in range(1, ngp + 1):
        os.makedirs(tmp_path / str(g))
    s.step()
    s.particles_write(str(tmp_path), ngp, istep=2)
    s.step()
    s.particles_write(str(tmp_path), ngp, istep=3, append=True)
    pos, vel = s.particles_get()
    t = s.time_info()["time"]
    for g in range(1, ngp + 1):
        for kind, arr in (("pvel", vel), ("ppos", pos)):
            recs = _records(tmp_path / str(g) / f"{kind}1g{g}_s0")
            assert struct.unpack(">4i", recs[0]) == (4 * nrefp, nrefp, 4, 3)
            assert len(recs) == 1 + 2 * (1 + 3 * 4)
            last = recs[1 + 13:]
            step, time = struct.unpack(">id", last[0])
            assert step == 2 and time == t
            for comp in range(3):
                sets = [np.frombuffer(last[1 + 4 * comp + k], dtype=">f8") for k in range(4)]
                np.testing.assert_array_equal(sets[0], arr[:nrefp, comp])
                for ii in range(1, 4):
                    i0 = nrefp + ((g - 1) * 3 + ii - 1) * nrefp
                    np.testing.assert_array_equal(sets[ii], arr[i0:i0 + nrefp, comp])
    s.close()
