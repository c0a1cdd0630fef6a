"""The oracle against the reference's OWN CPU dual contouring backend (CpuDualContouringBackend::
extract, src/cpp/dc_backend.cpp:51-125 through contouring.cpp, Cell.cpp and hermite_update.cpp),
compiled from the reference's sources into oracle/_ref/ref_cpu_dc with stand-in Eigen headers
(oracle/ref_eigen/: JacobiSVD restated as a one-sided Jacobi SVD). Skipped where the program was
not built (no reference tree). The bar: identical vertex count and active-cell count, identical
quads (order and winding), every vertex the float rounding of the oracle's FP64 vertex (within
FP64 noise: the two 3x3 SVDs round differently). Cases: the reference's own dc_tests.cpp grids
(src/cpp/dc_tests.cpp:14-215), the CLI generators, sharp-feature CSG, smooth perturbed
spheres, exact zeros, ragged and minimal grids, anisotropic spacing."""
import os

import numpy as np
import pytest

import oracle as O

HAVE = os.path.exists(os.path.join(os.path.dirname(O.__file__), "_ref", "ref_cpu_dc"))
pytestmark = pytest.mark.skipif(not HAVE, reason="oracle/_ref/ref_cpu_dc was not built (no reference tree)")


def _cases():
    from contouring_b200 import synth
    return {
        # dc_tests.cpp: sphere 32^3 r=0.5, box 32^3, plane z 16^3, thin gap 32^3, +1 and -1 16^3
        "sphere32": lambda: synth.cli_sphere(32),
        "box32": lambda: synth.cli_box(32),
        "plane16": lambda: synth.cli_plane(16),
        "thin_gap32": lambda: synth.thin_gap(32),
        "empty16": lambda: synth.constant(16, 1.0),
        "full16": lambda: synth.constant(16, -1.0),
        "zeros16": lambda: synth.constant(16, 0.0),
        "cli_sphere48": lambda: synth.cli_sphere(48),
        "sphere48_r035": lambda: synth.sphere(48, 0.35),
        "csg48": lambda: synth.csg(48, seed=0),
        "csg40_seed3": lambda: synth.csg(40, seed=3),
        "rbf_sphere40": lambda: synth.rbf_sphere(40),
        "thin_shell40": lambda: synth.thin_shell(40),
        "noise20": lambda: synth.noise((20, 20, 20), seed=1),
        "noise_zeros17x23x9": lambda: synth.noise((17, 23, 9), seed=2, zero_frac=0.3),
        "noise_zeros_half": lambda: synth.noise((24, 19, 21), seed=3, zero_frac=0.5),
        "ternary": lambda: synth.ternary((21, 22, 23), seed=4),
        "plane17_zero_layer": lambda: synth.cli_plane(17),
        "sphere_zero_shell": lambda: synth.sphere_with_zero_shell(40),
        "tiny2x2x2": lambda: synth.noise((2, 2, 2), seed=9),
        "ragged3x2x5": lambda: synth.noise((3, 2, 5), seed=7),
        "ragged33x7x4": lambda: synth.noise((33, 7, 4), seed=44),
    }


def _check(vals, dims, sp, org, name):
    vals = vals.numpy() if hasattr(vals, "numpy") else np.asarray(vals)
    rV, rF, ractive = O.ref_cpu_extract(vals, dims, sp, org)
    r = O.dc_extract(vals, dims, sp, org, threads=0)
    assert len(rV) == len(r["V"]) == ractive == len(r["cells"]), name
    assert np.array_equal(rF, r["F"]), "%s: quads differ from the reference CPU backend's" % name
    if len(rV):
        tol = np.maximum(1.2e-7 * np.abs(r["V"]), 1e-9 * np.asarray(sp, np.float64))
        bad = np.abs(rV.astype(np.float64) - r["V"]) > tol
        assert not bad.any(), "%s: %d vertex coordinates beyond one float rounding" % (name, int(bad.sum()))
    return len(rV), len(rF)


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_oracle_matches_reference_cpu_backend(name):
    _check(*_cases()[name](), name)


def test_anisotropic_spacing_and_offset_origin():
    from contouring_b200 import synth
    vals, dims, sp, org = synth.noise((19, 14, 11), seed=12)
    _check(vals, dims, (0.05, 0.11, 0.031), (-0.73, 0.2, 1.5), "anisotropic")


def test_tiny_differences_and_far_origin():
    """A plane whose values differ by less than 1e-6 along z (the lerp parameter is then formed
    in double, Cell.cpp:49-52) on a grid placed far from the origin, where the float positions
    origin + i * spacing round (dc_backend.cpp:63-65)."""
    n = (13, 11, 16)
    k = np.arange(n[2], dtype=np.float64)[:, None, None]
    j = np.arange(n[1], dtype=np.float64)[None, :, None]
    i = np.arange(n[0], dtype=np.float64)[None, None, :]
    vals = (1e-7 * (k - 7.3) + 2e-9 * np.sin(i + 2.0 * j)).astype(np.float32) * np.ones((1, n[1], n[0]), np.float32)
    _check(vals.reshape(-1), n, (0.0625, 0.0625, 0.0625), (1000.25, -2048.5, 333.3), "tiny_far")


@pytest.mark.parametrize("seed", [5, 6, 7, 8])
def test_csg_seeds(seed):
    from contouring_b200 import synth
    _check(*synth.csg(28, seed=seed), "csg28_seed%d" % seed)
