"""Writes tests/golden/serde_fixture_digests.json: the length and SHA-256 of
the crate's two on-disk format fixtures (mesh_to_sdf/tests/sdf_generic_v1.bin
and sdf_grid_v1.bin, written by serde.rs:298-369).  The digests let
tests/test_serde.py check the library's bytes against the crate's on any
machine, without a copy of the fixtures.

    python tests/golden/make_serde_digests.py <reference checkout>
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    out = {}
    for name in ("sdf_generic_v1.bin", "sdf_grid_v1.bin"):
        with open(os.path.join(ref_root, "mesh_to_sdf", "tests", name), "rb") as f:
            data = f.read()
        out[name] = {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
    with open(os.path.join(HERE, "serde_fixture_digests.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(out)


if __name__ == "__main__":
    main(sys.argv[1])
