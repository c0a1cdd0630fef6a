"""The sparse (brick) backends on the GPU (B200SparseDualContouringBackend / ...Mvdc..., the
reference's CudaSparseDualContouringBackend and CudaSparseMvdcDualContouringBackend) against
  * the float CPU restatement (oracle/sparse_oracle.cpp): vertices, faces, active cells and
    every counter identical, bit for bit;
  * the reference's own sparse CUDA code built without FMA contraction (oracle/_ref,
    libref_sparse_exact.so): vertices, faces and counters identical, bit for bit — this pins
    the restatement to the reference itself;
  * the reference as shipped (nvcc's default FMA contraction): the same counts, vertices within
    1e-5 cell widths where the topology agrees (reported).
Grids: a smooth sphere, a sharp-feature CSG, thin shells (thin edges, two-vertex cells), a
ragged box and random values with exact zeros; brick sizes 1, 3, 8, 16; all normal modes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backends():
    from contouring_b200 import B200SparseDualContouringBackend
    b = {False: B200SparseDualContouringBackend(), True: B200SparseDualContouringBackend(multi_vertex_cells=True)}
    yield b
    for x in b.values():
        x.close()


def _grid(name):
    import torch
    from contouring_b200 import synth
    if name == "sphere32":
        return synth.sphere(32, radius=0.35)
    if name == "csg48":
        return synth.csg(48, seed=3)
    if name.startswith("shell48_"):
        return synth.thin_shell(48, seed=int(name[-1]))
    if name == "ragged":
        v, dims, sp, org = synth.rbf_sphere(44, seed=2)
        g = v.numpy().reshape(44, 44, 44)[2:39, 5:44, 0:29]       # (z, y, x) = (37, 39, 29)
        return torch.from_numpy(np.ascontiguousarray(g).reshape(-1)), (29, 39, 37), sp, org
    if name == "noise":
        return synth.noise((13, 11, 9), seed=5, scale=0.1, zero_frac=0.2)
    raise KeyError(name)


CASES = [("sphere32", 8, 0), ("csg48", 8, 0), ("csg48", 3, 1), ("csg48", 16, 2), ("shell48_0", 8, 0),
         ("shell48_1", 8, 1), ("ragged", 8, 0), ("ragged", 5, 1), ("noise", 1, 0), ("noise", 4, 1)]


def _run(be, vals, dims, sp, org, brick, mode):
    be.brick_size = brick
    be.normal_mode = mode
    V, F, st = be.extract_tensor(vals, dims, sp, org)
    return V.cpu().numpy(), F.cpu().numpy(), st, be.active_cells()


def _stats(st):
    return {"total_bricks": st.total_bricks, "active_bricks": st.active_bricks, "active_cells": st.active_cells,
            "qef_fallbacks": st.qef_fallback_count, "clamps": st.clamp_count, "invalid": st.invalid_count,
            "ambiguous_cells": st.ambiguous_cells, "multi_vertex_cells": st.multi_vertex_cells,
            "one_vertex_cells": st.one_vertex_cells, "two_vertex_cells": st.two_vertex_cells,
            "split_rejections": st.split_rejection_count, "faces_skipped": st.faces_skipped_due_to_missing_cluster}


@pytest.mark.parametrize("mvdc", [False, True])
@pytest.mark.parametrize("name,brick,mode", CASES)
def test_matches_oracle_and_reference(backends, name, brick, mode, mvdc):
    import oracle as O
    vals, dims, sp, org = _grid(name)
    d = vals.cuda()
    V, F, st, cells = _run(backends[mvdc], d, dims, sp, org, brick, mode)
    r = O.sparse_extract(vals.numpy(), dims, sp, org, brick_size=brick, mvdc=mvdc, normal_mode=mode)
    print("%s brick %d mode %d mvdc %d: %d vertices, %d faces, %s" % (
        name, brick, mode, mvdc, len(V), len(F), {k: v for k, v in r["stats"].items() if v}))
    assert np.array_equal(F, r["F"]), "faces differ from the restatement"
    assert np.array_equal(V.view(np.uint32), r["V"].view(np.uint32)), "vertices differ from the restatement"
    per_vertex_cell = np.repeat(r["cells"], np.diff(np.append(r["vstart"], len(r["V"]))))
    assert np.array_equal(cells, per_vertex_cell)
    assert _stats(st) == r["stats"]
    ref = O.ref_sparse(d.data_ptr(), dims, sp, org, brick_size=brick, normal_mode=mode, mvdc=mvdc, exact=True)
    if ref is None:
        pytest.skip("oracle/_ref/libref_sparse_exact.so was not built")
    assert np.array_equal(F, ref["F"]), "faces differ from the reference (no FMA)"
    assert np.array_equal(V.view(np.uint32), ref["V"].view(np.uint32)), "vertices differ from the reference (no FMA)"
    for k, v in r["stats"].items():
        assert ref["stats"][k] == v, k


@pytest.mark.parametrize("mvdc", [False, True])
@pytest.mark.parametrize("name", ["csg48", "shell48_0"])
def test_close_to_shipped_reference(backends, name, mvdc):
    """Against the reference built as shipped (FMA contraction): report how far apart."""
    import oracle as O
    vals, dims, sp, org = _grid(name)
    d = vals.cuda()
    V, F, st, _ = _run(backends[mvdc], d, dims, sp, org, 8, 0)
    ref = O.ref_sparse(d.data_ptr(), dims, sp, org, mvdc=mvdc, exact=False)
    if ref is None:
        pytest.skip("oracle/_ref/libref_sparse.so was not built")
    same_topo = len(V) == len(ref["V"]) and np.array_equal(F, ref["F"])
    err = np.abs(V.astype(np.float64) - ref["V"]).max() / sp[0] if len(V) == len(ref["V"]) else np.inf
    print("%s mvdc %d: ours %d/%d, shipped reference %d/%d vertices/faces, same topology %s, max vertex diff %.3g cells" % (
        name, mvdc, len(V), len(F), len(ref["V"]), len(ref["F"]), same_topo, err))
    assert abs(len(V) - len(ref["V"])) <= 0.002 * len(V) + 2
    assert abs(len(F) - len(ref["F"])) <= 0.002 * len(F) + 2
    if same_topo:
        assert err <= 1e-3


def test_host_path_and_device_path_agree(backends):
    from contouring_b200 import DenseSdfGrid
    vals, dims, sp, org = _grid("shell48_1")
    be = backends[True]
    be.brick_size, be.normal_mode = 8, 0
    mesh, st = be.extract(DenseSdfGrid(*dims, *sp, *org, values=vals.numpy()))
    V, F, st2, _ = _run(be, vals.cuda(), dims, sp, org, 8, 0)
    assert np.array_equal(mesh.vertices.reshape(-1, 3), V) and np.array_equal(mesh.faces.reshape(-1, 4), F)
    assert st.two_vertex_cells == st2.two_vertex_cells > 0


def test_rejections(backends):
    import torch
    from contouring_b200 import DcbError
    vals, dims, sp, org = _grid("sphere32")
    be = backends[False]
    be.brick_size = 0
    with pytest.raises(DcbError):
        be.extract_tensor(vals.cuda(), dims, sp, org)
    be.brick_size = 8
    be.options.emit_triangles = True
    try:
        with pytest.raises(DcbError):
            be.extract_tensor(vals.cuda(), dims, sp, org)
    finally:
        be.options.emit_triangles = False
    V, F, st = be.extract_tensor(vals.cuda(), dims, sp, org)
    with pytest.raises(DcbError):                      # the adjoint covers the dense path only
        be.backward_tensor(vals.cuda(), dims, sp, org, torch.zeros_like(V))


def test_empty_and_constant(backends):
    from contouring_b200 import synth
    for value in (1.0, -1.0):
        vals, dims, sp, org = synth.constant(16, value)
        for mvdc in (False, True):
            V, F, st, _ = _run(backends[mvdc], vals.cuda(), dims, sp, org, 8, 0)
            assert len(V) == 0 and len(F) == 0 and st.active_bricks == 0
