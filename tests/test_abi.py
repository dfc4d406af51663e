"""CPU tests of the C ABI and host logic (no GPU compute): the library loads, exports every symbol
include/*.h declares, and rejects bad arguments before touching the device."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from gamer_b200 import fluid, ic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(gb_\w+)\s*\(", src, flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(fluid.LIB_PATH):
        from gamer_b200 import build
        build.build()
    return fluid.load_library()


def test_header_declares_api():
    names = _declared_symbols()
    assert "gb_fluid_solve_device" in names and "gb_fluid_solve_host" in names
    assert set(fluid.EXPORTED) <= set(names)


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in _declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_strerror_and_version(lib):
    assert lib.gb_fluid_strerror(0) == b"success"
    assert lib.gb_fluid_strerror(-2) == b"array not 16-byte aligned"
    assert lib.gb_fluid_version() >= 100


@pytest.mark.parametrize("bad", [dict(lr_scheme=7), dict(rsolver=6), dict(precision=3), dict(flu_nxt=18),
                                 dict(flu_nxt=21), dict(gamma=1.0), dict(dual_energy=2)])
def test_create_rejects_bad_config_without_device(lib, bad):
    c = dict(scheme=3, lr_scheme=1, rsolver=4, precision=0, dual_energy=0, flu_nxt=20, gamma=5 / 3)
    c.update(bad)
    cfg = fluid._Config(c["scheme"], c["lr_scheme"], c["rsolver"], c["precision"], c["dual_energy"],
                        c["flu_nxt"], c["gamma"])
    h = ctypes.c_void_p()
    assert lib.gb_fluid_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    assert not h.value


@pytest.mark.parametrize("over,code", [(dict(lr_scheme=2), -1), (dict(lr_scheme=2, flu_nxt=26), -5),
                                       (dict(char_reconstruction=2), -1)])
def test_create_rejects_char_reconstruction_not_built(lib, over, code):
    """Characteristic limiting is built for every scheme and window the scheme takes: MHM+PPM on a
    window narrower than its FLU_NXT = 22 is invalid, one wider than 24 not built, and a flag other
    than 0 / 1 invalid."""
    c = dict(scheme=3, lr_scheme=1, rsolver=4, precision=0, dual_energy=0, flu_nxt=20, gamma=5 / 3,
             char_reconstruction=1)
    c.update(over)
    cfg = fluid._Config(c["scheme"], c["lr_scheme"], c["rsolver"], c["precision"], c["dual_energy"],
                        c["flu_nxt"], c["gamma"], c["char_reconstruction"])
    h = ctypes.c_void_p()
    assert lib.gb_fluid_create(ctypes.byref(cfg), ctypes.byref(h)) == code
    assert not h.value


@pytest.mark.parametrize("over", [dict(dual_energy=1), dict(flu_nxt=22), dict(lr_scheme=2, flu_nxt=24)])
def test_mhd_with_mhm_options_not_built(lib, over):
    """MHD with the MHM scheme (HLLD) is built on the scheme's own FLU_NXT (PLM 20, PPM 22) without
    dual energy: dual energy and the wider window are reported as not built."""
    c = dict(scheme=3, lr_scheme=1, rsolver=5, precision=0, dual_energy=0, flu_nxt=20, gamma=5 / 3)
    c.update(over)
    cfg = fluid._Config(c["scheme"], c["lr_scheme"], c["rsolver"], c["precision"], c["dual_energy"],
                        c["flu_nxt"], c["gamma"])
    h = ctypes.c_void_p()
    assert lib.gb_fluid_create(ctypes.byref(cfg), ctypes.byref(h)) == -5
    assert not h.value


def test_null_arguments_rejected(lib):
    assert lib.gb_fluid_create(None, None) == -1
    assert lib.gb_fluid_destroy(None) == -1
    p = fluid.SolverParams(dt=1e-3, dh=1e-2).c()
    assert lib.gb_fluid_solve_device(None, None, None, None, None, None, None, None, None, 1, ctypes.byref(p), None) == -1
    assert lib.gb_fluid_solve_host(None, None, None, None, None, None, None, None, 1, ctypes.byref(p)) == -1


def test_product_never_imports_the_oracle():
    for path in glob.glob(os.path.join(ROOT, "gamer_b200", "**", "*.*"), recursive=True):
        if path.endswith((".py", ".cu", ".cuh", ".h")):
            txt = open(path).read()
            assert "pyoracle" not in txt and "gamer_oracle" not in txt and "libgref" not in txt, path


def test_cut_and_assemble_round_trip():
    box = ic.lognormal_box(2, seed=1)
    pgs = ic.cut_patch_groups(box, 20)
    assert pgs.shape == (8, 5, 20, 20, 20)
    back = ic.assemble_box(pgs[:, :, 2:18, 2:18, 2:18], 2)
    assert np.array_equal(back, box)
    # the ghost zones wrap periodically: left ghost of PG (0,0,0) = right edge of PG (1,0,0)
    assert np.array_equal(pgs[0][:, 2:18, 2:18, 0:2], pgs[1][:, 2:18, 2:18, 16:18])


def test_ic_generators_physical():
    for box in (ic.lognormal_box(1, 0), ic.kelvin_helmholtz_box(1, 0), ic.blast_box(1, 0, dual=False),
                ic.acoustic_wave_box(1)):
        rho = box[0]
        ek = 0.5 * (box[1] ** 2 + box[2] ** 2 + box[3] ** 2) / rho
        assert (rho > 0).all() and (box[4] - ek > 0).all()


def test_ctypes_structs_match_the_header(tmp_path):
    """The Python mirrors of the header's structs have the C sizes and field offsets: a program
    compiled against include/gamer_b200_fluid.h prints them (gcc, no device)."""
    src = tmp_path / "layout.c"
    mirrors = {"gb_fluid_config": fluid._Config, "gb_fluid_params": fluid._Params,
               "gb_close_params": fluid._CloseParams}
    fields = "".join(f" P({t}, {f});" for t, m in mirrors.items() for f, _ in m._fields_)
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "gamer_b200_fluid.h"\n'
        "#define P(T, F) printf(\"%s.%s %zu\\n\", #T, #F, offsetof(T, F))\n"
        "int main(void) {\n"
        " printf(\"gb_fluid_config %zu\\n\", sizeof(gb_fluid_config));\n"
        " printf(\"gb_fluid_params %zu\\n\", sizeof(gb_fluid_params));\n"
        " printf(\"gb_close_params %zu\\n\", sizeof(gb_close_params));\n"
        f"{fields}\n"
        " return 0; }\n")
    exe = tmp_path / "layout"
    import subprocess
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    c = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                     check=True).stdout.splitlines())
    assert int(c["gb_fluid_config"]) == ctypes.sizeof(fluid._Config)
    assert int(c["gb_fluid_params"]) == ctypes.sizeof(fluid._Params)
    assert int(c["gb_close_params"]) == ctypes.sizeof(fluid._CloseParams)
    # every field of every mirror, at the C offset
    for t, m in mirrors.items():
        for f, _ in m._fields_:
            assert int(c[f"{t}.{f}"]) == getattr(m, f).offset, (t, f)


def test_device_wrappers_reject_mismatched_arrays_before_any_launch():
    """The C ABI takes bare pointers, so the Python wrappers of the close and fix-up entry points
    check every array's shape and dtype first (no device needed to see the refusal)."""
    import torch
    s = object.__new__(fluid.FluidSolver)
    s.ncomp, s.flu_nxt, s.precision = 5, 20, "fp32"
    p = fluid.SolverParams(dt=1e-3, dh=1e-2)
    ok_in, ok_out = torch.zeros((2, 5, 20, 20, 20)), torch.zeros((2, 5, 16, 16, 16))
    with pytest.raises(ValueError, match="flu_in"):
        s.correct_unphysical_device(torch.zeros((2, 5, 22, 22, 22)), ok_out, p)
    with pytest.raises(ValueError, match="flux"):
        s.correct_unphysical_device(ok_in, ok_out, p, flux=torch.zeros((2, 9, 5, 16, 15)))
    with pytest.raises(ValueError, match="flu_out"):
        s.correct_unphysical_device(ok_in, torch.zeros((2, 5, 16, 16, 16), dtype=torch.float64), p)
    with pytest.raises(ValueError, match="has_flux"):
        s.flux_fixup_device(torch.zeros((3, 5, 8, 8, 8)), torch.zeros((3, 6, 5, 8, 8)),
                            torch.zeros((2, 6), dtype=torch.uint8), p)
    with pytest.raises(ValueError, match="flux"):
        s.flux_fixup_device(torch.zeros((3, 5, 8, 8, 8)), torch.zeros((3, 6, 6, 8, 8)),
                            torch.zeros((3, 6), dtype=torch.uint8), p)
