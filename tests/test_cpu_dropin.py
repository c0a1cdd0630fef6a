"""include/dc_b200.h — the B200 engine as an IDualContouringBackend of the reference — compiled
with g++ against the reference's own include/dc_backend.h and include/dc_cuda.h (the reference
tree comes from PHANTY_REFERENCE_SRC, or from the path build() found it at, recorded in
oracle/_ref/reference_root.txt; the test is skipped where neither exists). On a machine without
a GPU the compiled driver (oracle/_ref/ref_b200_drive) must fail cleanly through the class's
exception path instead of exiting from inside the library."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVE = os.path.join(ROOT, "oracle", "_ref", "ref_b200_drive")


def _reference_include():
    ref = os.environ.get("PHANTY_REFERENCE_SRC")
    rec = os.path.join(ROOT, "oracle", "_ref", "reference_root.txt")
    if not ref and os.path.exists(rec):
        ref = open(rec).read().strip()
    inc = os.path.join(ref or "", "include")
    if not ref or not os.path.exists(os.path.join(inc, "dc_backend.h")):
        pytest.skip("the reference's include/ is not available here")
    return inc


def test_dropin_header_compiles_against_reference_headers(tmp_path):
    inc = _reference_include()
    src = tmp_path / "use_dc_b200.cpp"
    src.write_text(
        '#include "dc_b200.h"\n'
        '#include <memory>\n'
        '// the reference selects its backend behind this interface (dc_cli.cpp:315-322)\n'
        'std::unique_ptr<IDualContouringBackend> make_b200() {\n'
        '    return std::make_unique<B200DualContouringBackend>(0, DCB_METHOD_DUAL_CONTOURING);\n'
        '}\n'
        'DualContouringMesh run(B200DualContouringBackend& b, const DenseSdfGridDevice& g, DualContouringStats& s) {\n'
        '    return b.extract_device(g, s);\n'
        '}\n')
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
           "-I" + inc, "-I/usr/local/cuda/include", str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_dropin_driver_fails_cleanly_without_gpu(tmp_path):
    import numpy as np
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: tests/test_gpu_dropin.py drives the class")
    if not os.path.exists(DRIVE):
        pytest.skip("oracle/_ref/ref_b200_drive was not built (no reference tree here)")
    from contouring_b200 import DenseSdfGrid, io, synth
    io.write_sdf(str(tmp_path / "g.sdf"), DenseSdfGrid.from_tuple(synth.cli_sphere(12)))
    r = subprocess.run([DRIVE, str(tmp_path / "g.sdf"), str(tmp_path / "o.bin")], capture_output=True, text=True)
    assert r.returncode == 3 and "B200DualContouringBackend" in r.stderr, (r.returncode, r.stderr)
