"""CPU checks of the C-ABI boundary: the library loads and exports every
function that include/*.h declares; host-only entry points (geometry,
default parameters, error reporting) work without a GPU."""
import ctypes
import glob
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*int\s+(psdns_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(gpu_mod):
    names = declared_functions()
    assert len(names) >= 10
    lib = ctypes.CDLL(gpu_mod.lib_path())
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert names <= set(gpu_mod.EXPORTS) | names


def test_geometry_entry_point(gpu_mod, oracle_mod):
    # kxn = min(n/2, (int)(n sqrt(2)/3) + 1) (init.f:29) for every compiled n
    for n in (16, 32, 48, 64, 96, 128, 256, 512, 1024):
        assert gpu_mod.geometry(n)["kxn"] == min(n // 2, int(n * np.sqrt(2) / 3) + 1)
    for n in (16, 48, 64, 96, 256):
        g = gpu_mod.geometry(n)
        o = oracle_mod.Oracle(n, 0.01, kshift=4)
        og = o.geometry()
        assert g["kxn"] == o.kxn and g["xz_tot"] == o.xz_tot
        np.testing.assert_array_equal(g["cut"], og["cut"])
        np.testing.assert_array_equal(g["colstart"], og["colstart"])
        np.testing.assert_array_equal(g["kymax"], og["kymax"])
        o.close()


def test_default_params_match_reference_input(gpu_mod):
    p = gpu_mod.default_params()
    # PSDNS/input: iseed 122929298, kshift record, cfl 3.77; input.f:268-269 sequences
    assert p.seed_input == 122929298 and p.ksran == 1 and p.kranf1 == 5 and p.kranf2 == 5
    assert abs(p.cfl - 3.77) < 1e-12


def test_init_rejects_bad_parameters_without_touching_a_device(gpu_mod):
    import pytest
    for kw in ({"n": 20}, {"kshift": 7}, {"seed_input": -1}, {"nx": 64, "ny": 32, "nz": 64},
               {"nc": 2}, {"nc": 1, "pr": 0.0}):
        p = gpu_mod.default_params(n=64)
        for k, v in kw.items():
            if k == "n":
                p.nx = p.ny = p.nz = v
            else:
                setattr(p, k, v)
        with pytest.raises(gpu_mod.PsdnsError):
            gpu_mod.Solver(p)
    assert gpu_mod.last_error() != ""
