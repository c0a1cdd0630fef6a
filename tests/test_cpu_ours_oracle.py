"""Checks of the refinement oracle (oracle/ours_oracle.cpp) on the CPU: the same result on one
thread and on all, the quad topology of the dual-contouring start, and on a sphere vertices
that move towards the surface."""
import numpy as np


def _sphere(res=24):
    from contouring_b200 import synth
    vals, dims, sp, org = synth.sphere(res, radius=0.35)
    return vals.numpy(), dims, sp, org


def test_thread_count_does_not_change_the_result():
    import oracle as O
    vals, dims, sp, org = _sphere()
    a = O.ours(vals, dims, sp, org, outer_iters=2, threads=1)
    b = O.ours(vals, dims, sp, org, outer_iters=2, threads=0)
    assert np.array_equal(a["V"], b["V"]) and np.array_equal(a["F"], b["F"])


def test_topology_is_the_extraction_s():
    import oracle as O
    vals, dims, sp, org = _sphere()
    r = O.ours(vals, dims, sp, org, outer_iters=2)
    d = O.dc_extract(vals, dims, sp, org)
    assert np.array_equal(r["cells"], d["cells"])
    assert np.array_equal(np.sort(np.sort(r["F"], 1), 0), np.sort(np.sort(d["F"], 1), 0))


def test_sphere_vertices_approach_the_surface():
    import oracle as O
    vals, dims, sp, org = _sphere(32)
    start = O.ours(vals, dims, sp, org, outer_iters=0)          # Hermite centroids
    r = O.ours(vals, dims, sp, org, outer_iters=3)
    e0 = np.abs(np.linalg.norm(start["V"], axis=1) - 0.35).mean()
    e3 = np.abs(np.linalg.norm(r["V"], axis=1) - 0.35).mean()
    assert e3 < 0.6 * e0, (e0, e3)
    assert np.isfinite(r["V"]).all()
