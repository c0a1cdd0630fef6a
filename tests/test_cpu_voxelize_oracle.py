"""The voxelize-first mesh -> SDF restatement (oracle/mts_oracle.cpp, mts_compute_voxelized;
src/cuda/mesh_to_sdf_cuda.cu:458-577, 764-832) pinned on the CPU by known answers: a closed
surface's voxel solid holds its inside and is empty at the border, points beyond the band
are -10 inside and +10 outside, an open patch encloses nothing, the band values equal the
plain conversion's band, and the voxel resolution is clamped to [32, 2048]."""
import numpy as np


def _sphere_scene():
    from contouring_b200 import synth
    V, F = synth.icosphere_scene(1, 3, seed=3, noise=0.0)
    return V, F, synth.mesh_grid(V, 96)


def test_closed_surface_solid_and_signs():
    import oracle as O
    V, F, (dims, sp, org) = _sphere_scene()
    out, st, solid = O.mesh_to_sdf_voxelized(V, F, dims, org, sp, voxel_res=48, return_solid=True)
    assert solid[0].sum() == 0 and solid[-1].sum() == 0 and solid[:, 0].sum() == 0 and solid[:, :, 0].sum() == 0
    c = np.asarray(V, np.float64).mean(axis=0)
    vox = np.array([(dims[a] * sp[a]) / 48 for a in range(3)], np.float64)
    ci = np.floor((c - np.array(org)) / vox).astype(int)
    assert solid[ci[2], ci[1], ci[0]] == 1                   # the centre of the sphere is solid
    far = np.abs(out) == 10.0
    nx, ny, nz = dims
    zz, yy, xx = np.meshgrid(*(np.arange(n) for n in (nz, ny, nx)), indexing="ij")
    p = np.stack([org[0] + xx * sp[0], org[1] + yy * sp[1], org[2] + zz * sp[2]], -1).reshape(-1, 3)
    r = np.linalg.norm(p - c, axis=1)
    radius = np.linalg.norm(np.asarray(V, np.float64) - c, axis=1).mean()
    inside = far & (r < 0.8 * radius)
    outside = far & (r > 1.2 * radius)
    assert inside.any() and outside.any()
    assert np.all(out[inside] == -10.0) and np.all(out[outside] == 10.0)
    assert st["exterior_filled"] == int(np.sum(out == 10.0) - np.sum((out == 10.0) & ~far))


def test_band_equals_plain_band():
    import oracle as O
    V, F, (dims, sp, org) = _sphere_scene()
    out, st = O.mesh_to_sdf_voxelized(V, F, dims, org, sp, voxel_res=64)
    idx = np.nonzero(np.abs(out) != 10.0)[0].astype(np.int64)
    band = O.mesh_band_values(V, F, dims, org, sp, idx)
    assert np.array_equal(out[idx], band)
    assert st["band_points"] == len(idx)


def test_open_patch_encloses_nothing():
    import oracle as O
    V = np.array([[-0.3, -0.3, 0.01], [0.3, -0.3, 0.01], [0.3, 0.3, 0.01], [-0.3, 0.3, 0.01]], np.float32)
    F = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    dims, sp, org = (33, 33, 33), (1 / 32, 1 / 32, 1 / 32), (-0.5, -0.5, -0.5)
    out, st, solid = O.mesh_to_sdf_voxelized(V, F, dims, org, sp, voxel_res=33, return_solid=True)
    assert not np.any(out == -10.0)
    # only the (dilated) shell of the patch is solid
    assert 0 < solid.sum() < 0.05 * solid.size


def test_resolution_clamped():
    import oracle as O
    V, F, (dims, sp, org) = _sphere_scene()
    a = O.mesh_to_sdf_voxelized(V, F, dims, org, sp, voxel_res=8, return_solid=True)
    b = O.mesh_to_sdf_voxelized(V, F, dims, org, sp, voxel_res=32, return_solid=True)
    assert a[2].shape == (32, 32, 32) and np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
