"""Writes the golden fixtures in this folder (run from the repository root after
``make -C oracle ref REFERENCE=<reference tree>``: ``python tests/golden/make_golden.py``). Each
``dc_<case>.npz`` holds the input grid and two outputs for it:
  * the reference's OWN CPU backend (CpuDualContouringBackend::extract, src/cpp/dc_backend.cpp:
    51-125, compiled from its sources into oracle/_ref/ref_cpu_dc with the stand-in Eigen
    headers of oracle/ref_eigen/): float32 vertices ``ref_V``, quads ``ref_F``, its
    ``ref_active`` count — the pin, which needs no reference tree at test time;
  * the oracle's (oracle/dc_oracle.cpp): FP64 vertices ``V``, quads ``F``, vertex cells ``cells``.
The script refuses to write a fixture on which the two disagree (quads, counts, or a vertex
beyond one float rounding)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "phanty-sdf-cuda_b200")]


def cases():
    from contouring_b200 import synth
    return {
        "cli_sphere24": synth.cli_sphere(24),
        "cli_box20": synth.cli_box(20),
        "thin_gap24": synth.thin_gap(24),
        "csg28": synth.csg(28, seed=0),
        "noise_zeros9x11x7": synth.noise((9, 11, 7), seed=2, zero_frac=0.3),
        "ternary8": synth.ternary((8, 8, 8), seed=4),
    }


def main():
    import oracle as O
    for name, (vals, dims, sp, org) in cases().items():
        v = vals.numpy().astype(np.float32)
        r = O.dc_extract(v, dims, sp, org, threads=1)
        ref = O.ref_cpu_extract(v, dims, sp, org)
        if ref is None:
            raise SystemExit("oracle/_ref/ref_cpu_dc is missing: make -C oracle ref REFERENCE=<reference tree>")
        rV, rF, ractive = ref
        assert np.array_equal(rF, r["F"]) and len(rV) == len(r["V"]) == ractive, name
        # one float rounding of the same FP64 vertex, up to FP64 noise in near-zero coordinates
        tol = np.maximum(1.2e-7 * np.abs(r["V"]), 1e-9 * np.asarray(sp, np.float64))
        assert np.all(np.abs(rV.astype(np.float64) - r["V"]) <= tol), name
        np.savez_compressed(os.path.join(HERE, "dc_%s.npz" % name), values=v, dims=np.array(dims, np.int32),
                            spacing=np.array(sp, np.float32), origin=np.array(org, np.float32),
                            V=r["V"], F=r["F"], cells=r["cells"], ref_V=rV, ref_F=rF, ref_active=np.int64(ractive))
        print(name, len(r["V"]), len(r["F"]))


if __name__ == "__main__":
    main()
