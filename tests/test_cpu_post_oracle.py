"""The oracle's mesh post-pass (oracle/post_oracle.cpp) pinned to the reference's own
postprocess_mesh (src/cpp/dc_backend.cpp:217-558): against the committed digests of its output
(tests/golden/post_digests.json, made by tests/golden/make_post_golden.py) and, where
oracle/_ref/libref_post.so was built from the reference's source, against it directly."""
import hashlib
import json
import os

import numpy as np
import pytest

import post_scenes as S

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "post_digests.json")) as f:
    GOLDEN = json.load(f)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", sorted(S.SMALL))
def test_oracle_matches_reference_digests(name):
    import oracle as O
    V, F = S.SMALL[name]()
    g = GOLDEN[name]
    assert digest(V, F) == g["input"], "scene input changed; regenerate the digests"
    for close, remove in S.FLAGS:
        Vo, Fo, st = O.postprocess_mesh(V, F, close, remove)
        want = g["%d%d" % (close, remove)]
        assert (Vo.shape[0], Fo.shape[0]) == (want["nv"], want["nf"])
        assert digest(Vo, Fo) == want["sha256"], (name, close, remove)
        assert (st["vertex_count"], st["face_count"]) == (want["nv"], want["nf"])


def _same(a, b):
    return (a[0].shape == b[0].shape and a[1].shape == b[1].shape
            and np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)) and np.array_equal(a[1], b[1]))


@pytest.mark.parametrize("name", sorted(S.LARGE))
def test_oracle_matches_reference_build(name):
    import oracle as O
    V, F = S.LARGE[name]()
    flags = [(1, 1)] if name == "tube_4096" else [(1, 1), (1, 0), (0, 1)]
    for close, remove in flags:
        r = O.ref_postprocess_mesh(V, F, close, remove)
        if r is None:
            pytest.skip("oracle/_ref/libref_post.so was not built (make -C oracle ref)")
        assert _same(O.postprocess_mesh(V, F, close, remove), r), (name, close, remove)


def test_no_flags_and_empty_meshes_pass_through():
    import oracle as O
    V, F = S.figure_eight()
    Vo, Fo, _ = O.postprocess_mesh(V, F, 0, 0)
    assert np.array_equal(Vo, V) and np.array_equal(Fo, F)
    Vo, Fo, _ = O.postprocess_mesh(V, F[:0], 1, 1)
    assert np.array_equal(Vo, V) and Fo.shape == (0, 4)


def test_stats_describe_the_scene():
    import oracle as O
    V, F = S.tube(64)
    _, _, st = O.postprocess_mesh(V, F, 1, 1)
    assert st["boundary_edges"] == 128 and st["loops_found"] == 2 and st["loops_filled"] == 2
    V, F = S.tube(4097)
    _, _, st = O.postprocess_mesh(V, F, 1, 0)
    assert st["loops_found"] == 2 and st["loops_filled"] == 0 and st["fill_vertices"] == 0
    V, F = S.floaters(32)
    _, Fo, st = O.postprocess_mesh(V, F, 0, 1)
    assert st["components"] == 3 and st["kept_faces"] == Fo.shape[0] < F.shape[0]


def _random_mesh(seed):
    """A small messy quad mesh: lattice vertices (so many coincide or lie within the weld step),
    random quads (some degenerate, many sharing edges in odd ways), plus a clean patch."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(8, 60))
    lattice = rng.integers(0, 5, size=(n, 3)).astype(np.float32) * np.float32(0.25)
    jitter = (rng.random((n, 3)).astype(np.float32) - np.float32(0.5)) * np.float32(2e-6)
    V = lattice + np.where(rng.random((n, 1)) < 0.3, jitter, np.float32(0))
    F = rng.integers(0, n, size=(int(rng.integers(4, 80)), 4)).astype(np.int32)
    Vp, Fp = S.figure_eight()
    return np.concatenate([V, Vp + np.float32(3)]).astype(np.float32), np.concatenate([F, Fp + n]).astype(np.int32)


@pytest.mark.parametrize("seed", range(40))
def test_oracle_matches_reference_on_random_meshes(seed):
    import oracle as O
    V, F = _random_mesh(seed)
    for close, remove in S.FLAGS:
        r = O.ref_postprocess_mesh(V, F, close, remove)
        if r is None:
            pytest.skip("oracle/_ref/libref_post.so was not built (make -C oracle ref)")
        assert _same(O.postprocess_mesh(V, F, close, remove), r), (seed, close, remove)
