"""CPU tests of the oracle (the FP64 restatement of the reference CPU backend): against the
independent Python restatement, against the committed golden fixtures, and on the known
answers the reference's own tests and the algorithm give (src/cpp/dc_tests.cpp:14-215)."""
import glob
import os

import numpy as np
import pytest

import oracle as O
import py_reference_dc as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _synth():
    from contouring_b200 import synth
    return synth


def _np(t):
    vals, dims, sp, org = t
    return vals.numpy(), dims, sp, org


SMALL = {
    "cli_sphere12": lambda s: s.cli_sphere(12),
    "cli_box12": lambda s: s.cli_box(12),
    "cli_plane10": lambda s: s.cli_plane(10),
    "csg16": lambda s: s.csg(16, seed=0),
    "csg14_seed5": lambda s: s.csg(14, seed=5),
    "thin_gap12": lambda s: s.thin_gap(12),
    "noise7x8x6": lambda s: s.noise((7, 8, 6), seed=1),
    "noise_zeros7x6x8": lambda s: s.noise((7, 6, 8), seed=2, zero_frac=0.3),
    "ternary7": lambda s: s.ternary((7, 7, 7), seed=4),
    "zero_shell14": lambda s: s.sphere_with_zero_shell(14),
    "rbf_sphere12": lambda s: s.rbf_sphere(12),
    "tiny2x2x2": lambda s: s.noise((2, 2, 2), seed=9),
    "ragged3x2x5": lambda s: s.noise((3, 2, 5), seed=7),
}


@pytest.mark.parametrize("name", list(SMALL))
def test_oracle_matches_python_restatement(name):
    """Same active cells, same quads (order and winding), vertices within 1e-9 cell widths:
    the two restatements differ only in their 3x3 solvers (cyclic Jacobi vs LAPACK SVD)."""
    vals, dims, sp, org = _np(SMALL[name](_synth()))
    V, F, cells = P.extract(vals, dims, sp, org)
    r = O.dc_extract(vals, dims, sp, org, threads=2)
    assert np.array_equal(cells, r["cells"])
    assert np.array_equal(F, r["F"])
    if len(V):
        assert np.abs(V - r["V"]).max() / min(sp) <= 1e-9


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "dc_*.npz"))),
                         ids=lambda p: os.path.basename(p)[3:-4])
def test_oracle_matches_golden(path):
    g = np.load(path)
    r = O.dc_extract(g["values"], tuple(g["dims"]), tuple(g["spacing"]), tuple(g["origin"]), threads=0)
    assert np.array_equal(r["cells"], g["cells"])
    assert np.array_equal(r["F"], g["F"])
    assert np.abs(r["V"] - g["V"]).max(initial=0.0) <= 1e-12


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "dc_*.npz"))),
                         ids=lambda p: os.path.basename(p)[3:-4])
def test_oracle_matches_reference_cpu_golden(path):
    """The committed output of the reference's OWN CPU backend (compiled from its sources,
    tests/golden/make_golden.py): identical quads (order and winding) and vertex count, and
    every vertex the float rounding of the oracle's FP64 vertex."""
    g = np.load(path)
    r = O.dc_extract(g["values"], tuple(g["dims"]), tuple(g["spacing"]), tuple(g["origin"]), threads=0)
    assert np.array_equal(r["F"], g["ref_F"])
    assert len(r["V"]) == len(g["ref_V"]) == int(g["ref_active"])
    tol = np.maximum(1.2e-7 * np.abs(r["V"]), 1e-9 * g["spacing"].astype(np.float64))
    assert np.all(np.abs(g["ref_V"].astype(np.float64) - r["V"]) <= tol)


def test_golden_fixtures_present():
    assert len(glob.glob(os.path.join(GOLDEN, "dc_*.npz"))) >= 6


@pytest.mark.parametrize("value", [1.0, -1.0, 0.0])
def test_constant_grids_are_empty(value):
    """dc_tests.cpp:171-215: +1 and -1 grids give no vertices and no faces (and so does 0:
    zeros are neither sign)."""
    r = O.dc_extract(*_np(_synth().constant(16, value)))
    assert len(r["V"]) == 0 and len(r["F"]) == 0 and r["stats"]["active_cells"] == 0


def test_plane_vertices_on_plane():
    """A linear field z: every vertex lies on the plane at the x,y centre of its cell's
    Hermite points; one vertex per column, one quad per interior z edge column."""
    vals, dims, sp, org = _np(_synth().cli_plane(16))
    r = O.dc_extract(vals, dims, sp, org)
    V = r["V"]
    assert len(V) == 15 * 15 and len(r["F"]) == 14 * 14
    assert np.abs(V[:, 2]).max() < 1e-12
    ax = (np.float32(org[0]) + np.arange(16, dtype=np.float32) * np.float32(sp[0])).astype(np.float64)
    ci = r["cells"] % 15
    assert np.allclose(V[:, 0], 0.5 * (ax[ci] + ax[ci + 1]), atol=1e-12)


def _closed_manifold(F):
    """Every directed edge of the quads appears exactly once and its reverse exactly once."""
    e = np.concatenate([np.stack([F[:, q], F[:, (q + 1) % 4]], 1) for q in range(4)])
    key = e[:, 0].astype(np.int64) * (1 << 32) + e[:, 1]
    rkey = e[:, 1].astype(np.int64) * (1 << 32) + e[:, 0]
    return len(np.unique(key)) == len(key) and np.array_equal(np.sort(key), np.sort(rkey))


@pytest.mark.parametrize("res", [24, 40, 48])
def test_sphere_closed_and_consistently_wound(res):
    """A sphere (radius off the grid points) contours to a closed, consistently oriented
    genus-0 quad mesh (V - E + F = 2) whose vertices lie within a cell width of the sphere."""
    vals, dims, sp, org = _np(_synth().cli_sphere(res))
    r = O.dc_extract(vals, dims, sp, org)
    V, F = r["V"], r["F"]
    assert _closed_manifold(F)
    assert len(V) - 2 * len(F) + len(F) == 2
    assert np.abs(np.linalg.norm(V, axis=1) - 0.5).max() < sp[0]


def test_thin_gap_one_connected_surface():
    """dc_tests.cpp:131-169: the union of two overlapping spheres (radius 0.25 at x = +-0.2)
    contours to one connected surface (dual contouring may pinch it along the crease where
    the spheres meet, so it need not be a manifold there)."""
    vals, dims, sp, org = _np(_synth().thin_gap(32))
    r = O.dc_extract(vals, dims, sp, org)
    F = r["F"]
    parent = np.arange(len(r["V"]))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a
    for q in F:
        for t in range(1, 4):
            ra, rb = find(q[0]), find(q[t])
            if ra != rb:
                parent[ra] = rb
    assert len({find(a) for a in range(len(parent))}) == 1


def test_vertex_count_equals_active_cells():
    """dc_tests.cpp:41-47: one vertex per active cell, all face indices in range, no NaN."""
    vals, dims, sp, org = _np(_synth().csg(40, seed=2))
    r = O.dc_extract(vals, dims, sp, org)
    st = r["stats"]
    assert st["active_cells"] == st["vertex_count"] == len(r["V"])
    assert st["face_count"] == len(r["F"])
    assert np.isfinite(r["V"]).all()
    assert r["F"].min() >= 0 and r["F"].max() < len(r["V"])
    assert np.all(np.diff(r["cells"]) > 0)


def test_threads_do_not_change_results():
    vals, dims, sp, org = _np(_synth().csg(36, seed=1))
    a = O.dc_extract(vals, dims, sp, org, threads=1)
    b = O.dc_extract(vals, dims, sp, org, threads=4)
    assert np.array_equal(a["V"], b["V"]) and np.array_equal(a["F"], b["F"])


def test_rejects_bad_shapes():
    with pytest.raises(ValueError):
        O.dc_extract(np.zeros(10, np.float32), (2, 2, 2), (1, 1, 1), (0, 0, 0))


def test_triangulate_splits_and_orients():
    """triangulate_v1 on the oracle's sphere: two triangles per quad along the a-c diagonal,
    each wound like its quad, so the triangle mesh is closed and consistently oriented."""
    vals, dims, sp, org = _np(_synth().cli_sphere(24))
    r = O.dc_extract(vals, dims, sp, org)
    T = O.triangulate(r["V"], r["F"])
    assert T.shape == (2 * len(r["F"]), 3)
    F = r["F"]
    assert np.array_equal(np.sort(T[0::2], 1), np.sort(F[:, [0, 1, 2]], 1))
    assert np.array_equal(np.sort(T[1::2], 1), np.sort(F[:, [0, 2, 3]], 1))
    e = np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]]).astype(np.int64)
    key = e[:, 0] * (1 << 32) + e[:, 1]
    assert len(np.unique(key)) == len(key)
    assert np.array_equal(np.sort(key), np.sort(e[:, 1] * (1 << 32) + e[:, 0]))


def test_triangulate_flips_against_the_quad_normal():
    """A quad whose second triangle folds back is flipped; a degenerate quad is left as is."""
    V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0.2, 0.1, 0.0]], np.float64)
    T = O.triangulate(V, np.array([[0, 1, 2, 3]]))
    assert T.tolist() == [[0, 1, 2], [0, 3, 2]]
    Z = np.zeros((4, 3))
    assert O.triangulate(Z, np.array([[0, 1, 2, 3]])).tolist() == [[0, 1, 2], [0, 2, 3]]


def test_negated_grid_flips_every_quad():
    """Negating every value keeps the active cells and the vertices (the normal equations see
    each normal twice, so its sign cancels; only lerp_t's +1e-16 moves the samples by ~1e-16)
    and reverses every quad's winding: the orientation test is dot(quad normal, gradient sum),
    and the gradients negate exactly (contouring.cpp:624-641)."""
    vals, dims, sp, org = _np(_synth().csg(32, seed=4))
    a = O.dc_extract(vals, dims, sp, org)
    b = O.dc_extract(-vals, dims, sp, org)
    assert np.array_equal(a["cells"], b["cells"])
    assert np.abs(a["V"] - b["V"]).max() <= 1e-9 * min(sp)
    assert len(a["F"]) == len(b["F"]) > 0
    assert np.array_equal(b["F"], a["F"][:, [0, 3, 2, 1]])


def test_power_of_two_scale_keeps_the_mesh():
    """Scaling every value by 4 keeps every sign, every lerp parameter (up to lerp_t's +1e-16)
    and every normal direction, so the same cells, quads and windings, and the vertices to
    ~1e-13 (contouring.cpp:486-741, Cell.cpp:49-52, 80-155)."""
    vals, dims, sp, org = _np(_synth().csg(32, seed=6))
    a = O.dc_extract(vals, dims, sp, org)
    b = O.dc_extract(vals * np.float32(4.0), dims, sp, org)
    assert np.array_equal(a["cells"], b["cells"])
    assert np.array_equal(a["F"], b["F"]) and len(a["F"]) > 0
    assert np.abs(a["V"] - b["V"]).max() <= 1e-9 * min(sp)
