"""The float restatement of the reference's sparse (brick) backends (oracle/sparse_oracle.cpp)
pinned on the CPU by known answers: empty constant grids, vertices on a plane, the multi-vertex
variant equal to the single-vertex one on a smooth surface, thin edges doubled into reversed
quads, and the same result on one thread and on all. Its bit-for-bit pin against the
reference's own CUDA code runs on the GPU (tests/test_gpu_sparse.py)."""
import numpy as np
import pytest


def _O():
    import oracle as O
    return O


def _synth():
    from contouring_b200 import synth
    return synth


@pytest.mark.parametrize("value", [1.0, -1.0])
@pytest.mark.parametrize("mvdc", [False, True])
def test_constant_grids_are_empty(value, mvdc):
    v, d, sp, org = _synth().constant(16, value)
    r = _O().sparse_extract(v.numpy(), d, sp, org, mvdc=mvdc)
    assert len(r["V"]) == 0 and len(r["F"]) == 0 and r["stats"]["active_bricks"] == 0


def test_plane_vertices_on_plane():
    """value = z - c with c between grid planes: every vertex that a face uses lies on z = c
    (all normals (0,0,1), one retained eigenvalue); cells that are only near zero get the
    cell centre and no face."""
    n = 20
    ax = np.float32(-1) + np.arange(n, dtype=np.float32) * np.float32(2.0 / (n - 1))
    c = np.float32(0.0371)
    Z = np.broadcast_to(ax[:, None, None], (n, n, n))
    v = (Z - c).astype(np.float32).reshape(-1)
    sp = (float(ax[1] - ax[0]),) * 3
    org = (float(ax[0]),) * 3
    for mvdc in (False, True):
        r = _O().sparse_extract(v, (n, n, n), sp, org, mvdc=mvdc)
        used = np.unique(r["F"])
        assert len(r["F"]) == (n - 1 - 1) ** 2
        assert np.abs(r["V"][used, 2] - c).max() <= 2e-7
        assert r["stats"]["two_vertex_cells"] == 0


def test_mvdc_equals_single_vertex_on_smooth_sphere():
    v, d, sp, org = _synth().sphere(32, radius=0.35)
    a = _O().sparse_extract(v.numpy(), d, sp, org, mvdc=False)
    b = _O().sparse_extract(v.numpy(), d, sp, org, mvdc=True)
    assert b["stats"]["two_vertex_cells"] == 0
    assert np.array_equal(a["V"], b["V"]) and np.array_equal(a["F"], b["F"])


def test_thin_edges_emit_reversed_pairs():
    v, d, sp, org = _synth().thin_shell(48, seed=0)
    r = _O().sparse_extract(v.numpy(), d, sp, org, mvdc=False)
    F = r["F"]
    rev = F[:, [0, 3, 2, 1]]
    # a thin edge's second quad is its first reversed, and comes right after it
    pairs = np.all(F[1:] == rev[:-1], axis=1)
    assert pairs.sum() > 100
    s = r["stats"]
    assert s["active_cells"] == len(r["cells"]) and len(r["V"]) == s["active_cells"]


def test_split_cells_have_two_vertices():
    v, d, sp, org = _synth().thin_shell(48, seed=1)
    r = _O().sparse_extract(v.numpy(), d, sp, org, mvdc=True)
    s = r["stats"]
    assert s["two_vertex_cells"] > 100
    assert len(r["V"]) == s["active_cells"] + s["two_vertex_cells"]
    counts = np.diff(np.append(r["vstart"], len(r["V"])))
    assert set(np.unique(counts)) <= {1, 2} and (counts == 2).sum() == s["two_vertex_cells"]
    assert s["one_vertex_cells"] + s["two_vertex_cells"] == s["active_cells"]


def test_thread_count_does_not_change_the_result():
    v, d, sp, org = _synth().csg(40, seed=3)
    a = _O().sparse_extract(v.numpy(), d, sp, org, mvdc=True, threads=1)
    b = _O().sparse_extract(v.numpy(), d, sp, org, mvdc=True, threads=0)
    assert np.array_equal(a["V"], b["V"]) and np.array_equal(a["F"], b["F"]) and a["stats"] == b["stats"]


def test_brick_culling_drops_near_zero_cells_without_a_sign_change():
    """A brick with no sign change contributes no cell, even where values are within
    0.45*vx of zero (mark_active_bricks_kernel tests signs only)."""
    n = 17
    v = np.full(n * n * n, 0.01, np.float32)          # all positive, all "near zero"
    sp = (0.1, 0.1, 0.1)
    r = _O().sparse_extract(v, (n, n, n), sp, (0.0, 0.0, 0.0))
    assert r["stats"]["active_bricks"] == 0 and len(r["V"]) == 0
    v.reshape(n, n, n)[0, 0, 0] = -0.01               # one negative corner: brick (0,0,0) only
    r = _O().sparse_extract(v, (n, n, n), sp, (0.0, 0.0, 0.0))
    assert r["stats"]["active_bricks"] == 1 and len(r["V"]) == 8 ** 3
