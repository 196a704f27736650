"""Generate the golden fixtures of tests/golden/ with the FP64 oracle.

The reference ships no golden vectors or known-answer tests and cannot be built
here (Fortran/MPI/FFTW), so these fixtures pin the oracle against regressions
(and the GPU path against the same numbers); they are not reference outputs.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402


def main():
    oracle.build()
    oracle.set_threads(1)
    n, nu, dt = 16, 0.02, 0.01
    kforce, tforce = 2.99, 0.5
    epsfor = 0.1 / (4.0 * (4.0 * np.pi / 3.0) * kforce ** 3)
    o = oracle.Oracle(n, nu, cfl=-1.0, dt=dt, kshift=1, seed_input=122929298)
    o.set_forcing(kforce, tforce, epsfor, 0.0)
    un0 = o.field_init(2468)
    o.set_state(un0)
    rng = np.random.default_rng(13579)
    pos0 = 1.0 + rng.random((64, 3)) * n
    o.particles_set(pos0)
    gsh = []
    for _ in range(3):
        assert o.step() == 0
        gsh.append(o.scalars()["gsh"])
    u, un = o.get_state()
    ek, dk, e6, st = o.spectra(1)
    tab, efkz = o.forcing()
    pos, vel = o.particles_get()
    np.savez_compressed(os.path.join(HERE, "rk2_forced_16.npz"),
                        n=n, viscos=nu, dt=dt, kforce=kforce, tforce=tforce, epsfor=epsfor, seed_field=2468,
                        seed_input=122929298, un0=un0, pos0=pos0, un=un, u=u, ek=ek, dk=dk,
                        stats=np.array([st[k] for k in ("tke", "eps", "skew", "klen", "kvel", "ktime", "ekl")]),
                        forcing=tab, efkz=efkz, pos=pos, vel=vel, gsh=np.array(gsh), rann2=o.rann2(5, 32))
    o.close()
    # geometry of the grids the scope table quotes
    geo = {}
    for m in (16, 64, 256, 1024):
        q = oracle.Oracle(m, 0.01, kshift=4)
        g = q.geometry()
        geo[f"cut_{m}"] = g["cut"]
        geo[f"xz_tot_{m}"] = q.xz_tot
        q.close()
    np.savez_compressed(os.path.join(HERE, "geometry.npz"), **geo)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
