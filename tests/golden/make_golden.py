"""Writes the oracle golden fixtures in this folder (run from the repository root:
``python tests/golden/make_golden.py``). Each ``dc_<case>.npz`` holds the input grid and the
oracle's output for it: FP64 vertices ``V``, quads ``F``, vertex cells ``cells``.

The oracle was first checked against the independent pure-Python restatement in
``tests/py_reference_dc.py`` on these grids (``tests/test_cpu_oracle.py`` repeats that check);
the fixtures then pin the oracle and the engine against regressions."""
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
        np.savez_compressed(os.path.join(HERE, "dc_%s.npz" % name), values=v, dims=np.array(dims, np.int32),
                            spacing=np.array(sp, np.float32), origin=np.array(org, np.float32),
                            V=r["V"], F=r["F"], cells=r["cells"])
        print(name, len(r["V"]), len(r["F"]))


if __name__ == "__main__":
    main()
