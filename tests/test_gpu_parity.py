"""B200 engine vs the CPU oracle (FP64 restatement of the reference CPU backend), through
the C ABI. Cases follow the reference's own tests (src/cpp/dc_tests.cpp:14-215) plus the
benchmark workloads at sizes the oracle finishes in seconds, and edge cases."""
import numpy as np
import pytest

from dc_compare import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from contouring_b200 import B200DualContouringBackend
    b = B200DualContouringBackend(0)
    yield b
    b.close()


def _cases():
    from contouring_b200 import synth
    return {
        # dc_tests.cpp cases
        "sphere32": lambda: synth.cli_sphere(32),
        "box32": lambda: synth.cli_box(32),
        "plane16": lambda: synth.cli_plane(16),
        "thin_gap32": lambda: synth.thin_gap(32),
        "empty16": lambda: synth.constant(16, 1.0),
        "full16": lambda: synth.constant(16, -1.0),
        # the CLI cross-check grid (dc_cli --generate sphere -g 128) and the small config
        "cli_sphere128": lambda: synth.cli_sphere(128),
        "sphere128_r035": lambda: synth.sphere(128, 0.35),
        # sharp features and perturbed smooth surfaces
        "csg96": lambda: synth.csg(96, seed=0),
        "csg128_seed3": lambda: synth.csg(128, seed=3),
        "rbf_sphere64": lambda: synth.rbf_sphere(64),
        # noise: dense activity, exact zeros (zeros are Hermite crossings but neither sign)
        "noise20": lambda: synth.noise((20, 20, 20), seed=1),
        "noise_zeros17x23x9": lambda: synth.noise((17, 23, 9), seed=2, zero_frac=0.3),
        "noise_zeros_half": lambda: synth.noise((24, 19, 21), seed=3, zero_frac=0.5),
        "ternary": lambda: synth.ternary((21, 22, 23), seed=4),
        # level set exactly on a grid plane (z = 0 at k = 8): no strictly mixed cell
        "plane17_zero_layer": lambda: synth.cli_plane(17),
        "sphere_zero_shell": lambda: synth.sphere_with_zero_shell(40),
    }


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_parity(backend, name):
    m = compare(backend, _cases()[name](), name)
    print(m)


def test_plane_vertices_exact(backend):
    """z = const plane: every vertex sits on the plane (contouring a linear field)."""
    from contouring_b200 import synth, DenseSdfGrid
    vals, dims, sp, org = synth.cli_plane(16)
    mesh, stats = backend.extract(DenseSdfGrid.from_tuple((vals, dims, sp, org)))
    V = mesh.vertices.reshape(-1, 3)
    assert stats.vertex_count == 15 * 15 and stats.face_count == 14 * 14
    assert np.abs(V[:, 2]).max() < 1e-6


def test_deterministic(backend):
    from contouring_b200 import synth, DenseSdfGrid
    g = DenseSdfGrid.from_tuple(synth.csg(96, seed=5))
    m1, _ = backend.extract(g)
    m2, _ = backend.extract(g)
    assert np.array_equal(m1.vertices, m2.vertices) and np.array_equal(m1.faces, m2.faces)


@pytest.mark.parametrize("dims", [(2, 2, 2), (3, 2, 5), (33, 7, 4), (5, 40, 3), (130, 3, 3)])
def test_odd_shapes(backend, dims):
    """Minimal and ragged grids, nx not a multiple of 4 (scalar load path)."""
    from contouring_b200 import synth
    compare(backend, synth.noise(dims, seed=sum(dims)), "noise%s" % (dims,))


def test_anisotropic_spacing(backend):
    from contouring_b200 import synth
    vals, dims, sp, org = synth.sphere(48, 0.3)
    compare(backend, (vals, dims, (sp[0], sp[1] * 1.5, sp[2] * 0.75), org), "anisotropic")


def test_force_fp64_matches_oracle_closely(backend):
    """Every cell on the FP64 path: vertices agree with the oracle to ~1e-12 cell widths."""
    from contouring_b200 import synth, DenseSdfGrid
    from dc_compare import run_oracle
    t = synth.csg(64, seed=1)
    backend.options.force_fp64 = True
    try:
        mesh, stats = backend.extract(DenseSdfGrid.from_tuple(t))
    finally:
        backend.options.force_fp64 = False
    ref = run_oracle(t)
    V = mesh.vertices.reshape(-1, 3).astype(np.float64)
    assert stats.escalated_fp64_cells == stats.vertex_count
    assert np.array_equal(mesh.faces.reshape(-1, 4), ref["F"])
    # float output rounding only: compare against the oracle rounded to float
    assert np.array_equal(V, ref["V"].astype(np.float32).astype(np.float64))


def test_invalid_arguments(backend):
    from contouring_b200 import DenseSdfGrid, DcbError
    with pytest.raises(DcbError):
        backend.extract(DenseSdfGrid(1, 4, 4, 0.1, 0.1, 0.1, 0, 0, 0, np.zeros(16, np.float32)))
    with pytest.raises(DcbError):
        backend.extract(DenseSdfGrid(4, 4, 4, 0.1, 0.1, 0.1, 0, 0, 0, np.zeros(10, np.float32)))
    with pytest.raises(DcbError):
        backend.extract(DenseSdfGrid(4, 4, 4, float("nan"), 0.1, 0.1, 0, 0, 0, np.zeros(64, np.float32)))


def _golden():
    import glob
    import os
    return sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dc_*.npz")))


@pytest.mark.parametrize("path", _golden(), ids=lambda p: p.rsplit("/", 1)[-1][3:-4])
def test_engine_matches_golden(backend, path):
    """The committed oracle fixtures, checked without running the oracle."""
    from contouring_b200 import DenseSdfGrid
    from dc_compare import VERTEX_TOL
    g = np.load(path)
    grid = DenseSdfGrid(*[int(x) for x in g["dims"]], *[float(x) for x in g["spacing"]],
                        *[float(x) for x in g["origin"]], values=g["values"])
    mesh, stats = backend.extract(grid)
    assert np.array_equal(backend.active_cells(), g["cells"])
    assert np.array_equal(mesh.faces.reshape(-1, 4), g["F"])
    V = mesh.vertices.reshape(-1, 3).astype(np.float64)
    if len(V):
        assert (np.abs(V - g["V"]) / g["spacing"].astype(np.float64)).max() <= VERTEX_TOL
    # the reference's own CPU backend's output on the same grid (compiled from its sources)
    assert np.array_equal(mesh.faces.reshape(-1, 4), g["ref_F"])
    assert stats.vertex_count == len(g["ref_V"]) == int(g["ref_active"])
    if len(V):
        assert (np.abs(V - g["ref_V"]) / g["spacing"].astype(np.float64)).max() <= VERTEX_TOL


@pytest.mark.parametrize("name", ["sphere32", "csg96", "noise_zeros17x23x9", "ternary", "sphere_zero_shell"])
def test_triangles_match_oracle(backend, name):
    """emit_triangles: triangulate_v1 of the quads, oriented from the FP64 vertices; the
    triangles equal the oracle's triangulation of its own quads exactly."""
    import oracle as O
    from contouring_b200 import DenseSdfGrid
    from dc_compare import run_oracle
    t = _cases()[name]()
    backend.options.emit_triangles = True
    try:
        mesh, stats = backend.extract(DenseSdfGrid.from_tuple(t))
        V2, F2, st2 = backend.extract_tensor(t[0].cuda(), t[1], t[2], t[3])
    finally:
        backend.options.emit_triangles = False
    ref = run_oracle(t)
    T = O.triangulate(ref["V"], ref["F"])
    assert stats.face_count == len(T) == 2 * len(ref["F"])
    assert np.array_equal(mesh.faces.reshape(-1, 3), T)
    assert np.array_equal(F2.cpu().numpy(), T)
