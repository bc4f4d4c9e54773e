"""Writes tests/golden/ingest_digests.json from the reference itself.

Run here, where the reference is compiled from its sources (oracle/_ref):
    python tests/golden/make_ingest_golden.py

For every case of tests/ingest_cases.py: the digest of the scene the
reference's parseConfig + buildScene (float build) makes from the config
(positions, triangles, materials, colours, views), and the triangle and
view counts.  The mesh files are written from seeded data into a
temporary directory, so the digests do not depend on where they lie.
"""
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main():
    from ref import ref_config
    import ingest_cases as cases
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, text in cases.configs(cases.write_meshes(d)).items():
            r = ref_config(text)
            out[name] = dict(digest=cases.digest(r["pos"], r["tris"], r["tri_mat"], r["mat_color"], r["views"]),
                             tris=int(len(r["tris"])), views=int(len(r["views"])))
    path = os.path.join(HERE, "ingest_digests.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print(path, len(out), "cases")


if __name__ == "__main__":
    main()
