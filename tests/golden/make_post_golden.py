"""Writes tests/golden/post_digests.json: for every small post-pass scene of tests/post_scenes.py
and every flag pair, the SHA-256 of the input and of the reference's own postprocess_mesh output
(src/cpp/dc_backend.cpp:217-558, built from its source into oracle/_ref/libref_post.so by
`make -C oracle ref`), with the output's counts. The oracle and the GPU post-pass are checked
against these digests where the reference sources are absent.

    python tests/golden/make_post_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"), os.path.join(ROOT, "phanty-sdf-cuda_b200")):
    sys.path.insert(0, p)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    import oracle as O
    import post_scenes as S
    out = {}
    for name, make in S.SMALL.items():
        V, F = make()
        entry = {"input": digest(V, F), "nv": int(V.shape[0]), "nf": int(F.shape[0])}
        for close, remove in S.FLAGS:
            r = O.ref_postprocess_mesh(V, F, close, remove)
            if r is None:
                raise SystemExit("oracle/_ref/libref_post.so is missing: run make -C oracle ref")
            entry["%d%d" % (close, remove)] = {"nv": int(r[0].shape[0]), "nf": int(r[1].shape[0]),
                                               "sha256": digest(r[0], r[1])}
        out[name] = entry
    with open(os.path.join(HERE, "post_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote %d scenes" % len(out))


if __name__ == "__main__":
    main()
