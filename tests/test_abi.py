"""The C-ABI library: builds for sm_100a, loads, exports every function that
include/mandor_b200.h declares, and fails loudly without a GPU (no CPU
path).  No compute call is made here."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for f in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(mg_[A-Za-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from mandor3_b200 import build
    build.build()
    import mandor3_b200
    return mandor3_b200.load()


def test_header_declares_the_stage_api():
    names = declared_functions()
    for n in ("mg_run_create", "mg_em_HHalfStep", "mg_em_energy", "mg_plasma_move",
              "mg_em_HStep", "mg_em_EStep_start", "mg_jbc_finish", "mg_em_EStep_finish",
              "mg_run_step", "mg_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_built_for_sm_100a(lib):
    from mandor3_b200 import build
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", build.LIB],
                         stdout=subprocess.PIPE, stderr=subprocess.STDOUT).stdout.decode()
    assert "sm_100a" in out


def test_version_string(lib):
    assert b"sm_100a" in lib.mg_version()


def test_no_cpu_fallback_without_a_device(lib):
    import mandor3_b200 as mg
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(mg.MandorError) as e:
        mg.Run((8, 8, 8), (0.1, 0.1, 0.1), 0.02, (0, 0, 0), (0, 0, 0))
    assert e.value.code in (-1, -2)


def test_bad_parameters_are_rejected_before_any_device_work(lib):
    import mandor3_b200 as mg
    with pytest.raises(mg.MandorError) as e:
        mg.Run((8, 8, 8), (0.1, 0.1, 0.1), 0.2, (0, 0, 0), (0, 0, 0))   # Courant > 1
    assert e.value.code == -2 and "unstable" in str(e.value)
    with pytest.raises(mg.MandorError) as e:
        mg.Run((8, 8, 8), (0.1, 0.1, 0.1), 0.02, (0, 1, 0), (0, 0, 0))  # half periodic
    assert e.value.code == -2


def test_estimate_bytes(lib):
    import mandor3_b200 as mg
    b = mg.estimate_bytes((256, 128, 128), (0.05,) * 3, 0.02, (2, 2, 2), (2, 2, 2), 4_500_000)
    assert 3e8 < b < 2e9
    # Without markers a run stepped alone keeps a second E and H set (six
    # more arrays of the padded grid) for its one-pass field step.
    n = (64, 48, 40)
    row = (4 + n[2] + 1 + 2 + 3) & ~3
    total = row * (n[1] + 5) * (n[0] + 5)
    b0 = mg.estimate_bytes(n, (0.05,) * 3, 0.02, (2, 2, 2), (2, 2, 2), 0)
    b1 = mg.estimate_bytes(n, (0.05,) * 3, 0.02, (2, 2, 2), (2, 2, 2), 1)
    assert b0 - b1 == 6 * total * 8 - 60          # less one FP64 marker's 60 bytes


# ctypes mirrors of the header's structures: same size and field offsets as
# the C compiler lays them out (a field added on one side only fails here).
STRUCTS = [("Params", "mg_params_t"), ("Laser", "mg_laser_t"), ("GaussSpot", "mg_gauss_spot_t"),
           ("Tfsf", "mg_tfsf_t"), ("Mirror", "mg_mirror_t"), ("TwoStream", "mg_two_stream_t"),
           ("DfUniform", "mg_df_uniform_t"), ("Maxwell", "mg_maxwell_t"), ("Foil", "mg_foil_t"),
           ("Place", "mg_place_t")]


def test_ctypes_structures_match_the_header(tmp_path):
    import mandor3_b200 as mg
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "mandor_b200.h"', 'int main (void) {']
    for py, c in STRUCTS:
        lines.append('printf ("%s size %%zu\\n", sizeof (%s));' % (py, c))
        for f, _ in getattr(mg, py)._fields_:
            lines.append('printf ("%s %s %%zu\\n", offsetof (%s, %s));' % (py, f, c, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], stdout=subprocess.PIPE, check=True).stdout.decode().split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for py, _ in STRUCTS:
        cls = getattr(mg, py)
        assert got[(py, "size")] == ctypes.sizeof(cls), py
        for f, _ in cls._fields_:
            assert got[(py, f)] == getattr(cls, f).offset, (py, f)
