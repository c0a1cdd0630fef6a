"""GPU mesh post-pass (dcb_post.cu through the C ABI) against the oracle's restatement of the
reference's postprocess_mesh (src/cpp/dc_backend.cpp:127-558) and the committed digests of the
reference's own output: vertices, faces and their order bit for bit, and the same counters."""
import hashlib
import json
import os

import numpy as np
import pytest

import post_scenes as S

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "post_digests.json")) as f:
    GOLDEN = json.load(f)
STATS = ("welded_vertices", "welded_faces", "components", "kept_faces", "boundary_edges", "loops_found",
         "loops_filled", "fill_vertices", "fill_faces", "vertex_count", "face_count")


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def backend():
    from contouring_b200 import B200DualContouringBackend
    return B200DualContouringBackend(device=0)


def run_gpu(backend, V, F, close, remove):
    import torch
    from contouring_b200 import postprocess_mesh_tensor
    Vo, Fo, st = postprocess_mesh_tensor(backend, torch.from_numpy(V).cuda(), torch.from_numpy(F).cuda(), close, remove)
    torch.cuda.synchronize()
    return Vo.cpu().numpy(), Fo.cpu().numpy(), st.as_dict()


def check_same(got, want, what):
    assert got[0].shape == want[0].shape and got[1].shape == want[1].shape, (what, got[0].shape, want[0].shape,
                                                                              got[1].shape, want[1].shape)
    assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32)), what
    assert np.array_equal(got[1], want[1]), what
    for k in STATS:
        assert got[2][k] == want[2][k], (what, k, got[2][k], want[2][k])


@pytest.mark.parametrize("name", sorted(S.SMALL))
def test_small_scenes_match_oracle_and_reference(backend, name):
    import oracle as O
    V, F = S.SMALL[name]()
    for close, remove in S.FLAGS:
        got = run_gpu(backend, V, F, close, remove)
        check_same(got, O.postprocess_mesh(V, F, close, remove), (name, close, remove))
        want = GOLDEN[name]["%d%d" % (close, remove)]
        assert digest(got[0], got[1]) == want["sha256"], (name, close, remove)


@pytest.mark.parametrize("name", sorted(S.LARGE))
def test_large_scenes_match_oracle(backend, name):
    import oracle as O
    V, F = S.LARGE[name]()
    flags = [(1, 1)] if name == "tube_4096" else [(1, 1), (1, 0), (0, 1)]
    for close, remove in flags:
        got = run_gpu(backend, V, F, close, remove)
        check_same(got, O.postprocess_mesh(V, F, close, remove), (name, close, remove))
        print("%s %d%d: %d/%d -> %d/%d, fill %d, %.3f ms" % (name, close, remove, V.shape[0], F.shape[0],
              got[0].shape[0], got[1].shape[0], got[2]["fill_vertices"], 0.0))


def test_engine_mesh_post_pass_on_device(backend):
    """A 160^3 extraction by the engine, post-processed where it lies, against the oracle."""
    import torch
    import oracle as O
    from contouring_b200 import postprocess_mesh_tensor
    vals, dims, sp, org = S._grid(160, lambda x, y, z: np.minimum(np.sqrt((x - 0.1) ** 2 + y * y + z * z) - 0.6,
                                                                  np.sqrt((x + 0.42) ** 2 + (y + 0.42) ** 2 + (z + 0.42) ** 2) - 0.04))
    V, F, _ = backend.extract_tensor(torch.from_numpy(vals).cuda(), dims, sp, org)
    Vh, Fh = V.cpu().numpy(), F.cpu().numpy()
    for close, remove in ((1, 1), (0, 1), (1, 0)):
        Vo, Fo, st = postprocess_mesh_tensor(backend, V, F, close, remove)
        got = (Vo.cpu().numpy(), Fo.cpu().numpy(), st.as_dict())
        check_same(got, O.postprocess_mesh(Vh, Fh, close, remove), ("engine160", close, remove))
    assert st.components == 0 and got[2]["loops_filled"] >= 5


def test_host_api_mirrors_reference_binding(backend):
    import oracle as O
    from contouring_b200 import DualContouringMesh, postprocess_mesh
    V, F = S.cut_sphere(24)
    m = postprocess_mesh(DualContouringMesh(V.reshape(-1), F.reshape(-1)), True, True, backend=backend)
    Vo, Fo, st = O.postprocess_mesh(V, F, 1, 1)
    assert np.array_equal(np.asarray(m.vertices).view(np.uint32), Vo.reshape(-1).view(np.uint32))
    assert np.array_equal(np.asarray(m.faces), Fo.reshape(-1))
    assert backend.last_postprocess_stats.loops_filled == st["loops_filled"]
    # neither flag: the input comes back unchanged
    m2 = postprocess_mesh(DualContouringMesh(V.reshape(-1), F.reshape(-1)), False, False, backend=backend)
    assert np.array_equal(np.asarray(m2.vertices), V.reshape(-1)) and np.array_equal(np.asarray(m2.faces), F.reshape(-1))


def test_invalid_meshes_are_refused(backend):
    from contouring_b200 import DcbError, DualContouringMesh, postprocess_mesh
    V, F = S.figure_eight()
    bad = F.copy()
    bad[3, 2] = V.shape[0]
    with pytest.raises(DcbError, match="out of range"):
        postprocess_mesh(DualContouringMesh(V, bad), True, True, backend=backend)
    Vn = V.copy()
    Vn[7, 1] = np.nan
    with pytest.raises(DcbError, match="non-finite"):
        postprocess_mesh(DualContouringMesh(Vn, F), True, True, backend=backend)
    # the handle stays usable
    m = postprocess_mesh(DualContouringMesh(V, F), True, True, backend=backend)
    assert len(m.faces) // 4 == 144


@pytest.mark.parametrize("seed", range(40))
def test_random_messy_meshes_match_oracle(backend, seed):
    """Lattice vertices (many coincide), random and degenerate quads, tangled boundaries."""
    import oracle as O
    from test_cpu_post_oracle import _random_mesh
    V, F = _random_mesh(seed)
    for close, remove in S.FLAGS:
        check_same(run_gpu(backend, V, F, close, remove), O.postprocess_mesh(V, F, close, remove), (seed, close, remove))
