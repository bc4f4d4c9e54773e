"""Scene-ingest cases shared by tests/test_ingest.py and
tests/golden/make_ingest_golden.py: mesh files written from seeded data and
configs that use them.

Every reference loader path is exercised: OBJ with texture/normal indices,
negative indices, polygons fanned into triangles, an out-of-range index,
CRLF lines and ignored records; PLY in ascii, binary little endian and
binary big endian, with extra properties, an extra element, both
vertex_indices and vertex_index lists and mixed numeric types; mesh
modifiers (scale, translate, color); every procedural scene; views from
view, orbit and walk lines; degenerate triangles (removed with their
materials)."""
from __future__ import annotations

import os
import struct

import numpy as np


def _verts(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.round(rng.uniform(-2, 2, (n, 3)), 4)


def write_meshes(d: str) -> dict:
    """Writes the mesh files into directory `d`; returns name -> path."""
    os.makedirs(d, exist_ok=True)
    paths = {}
    # OBJ: 8 vertices, texture and normal records, mixed face forms
    v = _verts(1, 8)
    lines = ["# seeded test mesh", "o thing", "g part"]
    lines += [f"v\t{x:.4f} {y:.4f}\t{z:.4f}" for x, y, z in v[:4]]
    lines += [f"v {x:.4f} {y:.4f} {z:.4f}\r" for x, y, z in v[4:]]
    lines += ["vt 0.5 0.5", "vn 0 0 1", "s off", "usemtl wood"]
    lines += ["f 1 2 3",                      # triangle
              "f 1/1/1 2/1/1 3/1/1 4/1/1",    # quad with texture and normal indices
              "f -4 -3 -2 -1",                # negative indices: the last four vertices
              "f 1//1 5//1 6//1 7//1 8//1",   # pentagon
              "f 1 2 99",                     # index out of range: dropped
              "f 2 2 3",                      # repeated index: degenerate, removed
              "  f 3 4 5\r",                  # leading blanks, CRLF
              "l 1 2"]
    paths["obj"] = os.path.join(d, "mixed.obj")
    with open(paths["obj"], "w", newline="") as f:
        f.write("\n".join(lines) + "\n")

    # PLY ascii: extra vertex properties, an extra element, vertex_indices
    v = _verts(2, 6)
    hdr = ["ply", "format ascii 1.0", "comment seeded", "element vertex 6", "property float x", "property float y",
           "property float z", "property float nx", "property uchar red", "element face 4",
           "property list uchar int vertex_indices", "element edge 1", "property int vertex1", "property int vertex2",
           "end_header"]
    body = [f"{x:.4f} {y:.4f} {z:.4f} 0.0 {i * 20}" for i, (x, y, z) in enumerate(v)]
    body += ["3 0 1 2", "4 0 2 3 4", "3 3 4 5", "3 1 5 7", "0 1"]
    paths["ply_ascii"] = os.path.join(d, "ascii.ply")
    with open(paths["ply_ascii"], "w") as f:
        f.write("\n".join(hdr + body) + "\n")

    # PLY binary little endian: float xyz plus a float property, uint vertex_index lists
    v = _verts(3, 7).astype(np.float32)
    hdr = ["ply", "format binary_little_endian 1.0", "element vertex 7", "property float x", "property float y",
           "property float z", "property float confidence", "element face 3",
           "property list uchar uint vertex_index", "end_header"]
    b = b"".join(struct.pack("<4f", *p, 0.5) for p in v)
    for face in ([0, 1, 2], [2, 3, 4, 5], [4, 5, 6, 0, 1]):
        b += struct.pack("<B", len(face)) + struct.pack(f"<{len(face)}I", *face)
    paths["ply_le"] = os.path.join(d, "le.ply")
    with open(paths["ply_le"], "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode() + b)

    # PLY binary big endian: double xyz, short property, int32 vertex_indices
    v = _verts(4, 5)
    hdr = ["ply", "format binary_big_endian 1.0", "element vertex 5", "property double x", "property double y",
           "property double z", "property short flags", "element face 3", "property list uint8 int32 vertex_indices",
           "end_header"]
    b = b"".join(struct.pack(">3dh", *p, -3) for p in v)
    for face in ([0, 1, 2], [1, 2, 3, 4], [0, 4, 9]):
        b += struct.pack(">B", len(face)) + struct.pack(f">{len(face)}i", *face)
    paths["ply_be"] = os.path.join(d, "be.ply")
    with open(paths["ply_be"], "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode() + b)
    return paths


def configs(p: dict) -> dict:
    """name -> config text (mesh paths from write_meshes)."""
    return {
        "plant": "# potted plant\nname plant\nmesh procedural plant\nup 0 1 0\nview 2.6 1.7 3.4  0 0.55 0  45\n"
                 "orbit 0 0.7 0  3.8 1.0 12 45\npoint_light 1.0 3.0 0.8\narea_light 0.9 2.8 0.7  0.4 0 0  0 0 0.4\n",
        "plant_seed11": "mesh procedural plant seed=11\n",
        "room": "name room\nmesh procedural room\ncull_backfaces 0\nup 0 1 0\norbit 4 1.2 4  2.8 0.7 8 70\n"
                "point_light 5.5 2.6 2.5\narea_light 4 2.95 4  1 0 0  0 0 1\n",
        "building_small": "mesh procedural building floors=2 rooms=3 detail=8\n"
                          "walk 1.0 4.6 17.5  39 4.4 17.5  12 70\npoint_light 2.5 5.6 18.5\n",
        "tess_sweep": "mesh procedural tess_sweep stacks=5\nview 0 4 9  0 0 0 50\n",
        "analytic": "mesh procedural analytic h=1.5 occ=0.7 ox=0.2 oz=-0.1 floor=6\n"
                    "area_light 0 3 0  1 0 0  0 0 1\nlight_intensity 2.5\nbackground 0.1 0.2 0.3\n",
        "random_tris": "mesh procedural random_tris n=40 seed=3 size=0.2\n",
        "sphere_floor": "mesh procedural sphere stacks=9 r=2\n"
                        "mesh procedural floorquad y=-2 size=7 scale 2 translate 1 2 3\n"
                        "up 0 0 1\norbit 0 0 0  5 1 5 50\ncull_backfaces 1\n",
        "obj": f"mesh obj {p['obj']} scale 2 translate 1 0 -1 color 0.2 0.3 0.4\nview 0 0 6  0 0 0 40\n",
        "ply_ascii": f"mesh ply {p['ply_ascii']}\n",
        "ply_le": f"mesh ply {p['ply_le']} scale 0.5\n",
        "ply_be": f"mesh ply {p['ply_be']} translate 0 1 0\n",
        "mixed": f"name mixed\nmesh obj {p['obj']}\nmesh ply {p['ply_ascii']}\nmesh procedural analytic\n"
                 f"mesh ply {p['ply_le']}\nmesh ply {p['ply_be']}\nmesh obj {p['obj']} color 1 0 0\n"
                 f"mesh ply {p['ply_ascii']} scale 3\n",
    }


# config text -> (a phrase of the reference's rejection, a phrase of ours):
# both sides reject the config for the same reason, each in its own words
ERRORS = {
    "bogus 1 2 3\n": ("unknown key 'bogus'", "line 1: 'bogus' is not a config key"),
    "view 1 2 3\n": ("expected 7 numbers after 'view'", "line 1: 'view' takes 7 numbers, got 3"),
    "mesh procedural room\nup 0 x 1\n": ("line 2", "line 2: 'x' is not a number"),
    "mesh stl part.stl\n": ("unknown mesh type stl", "mesh kind 'stl' is not obj, ply or procedural"),
    "mesh procedural teapot\n": ("unknown procedural scene 'teapot'", "no procedural scene named 'teapot'"),
    "mesh obj /nonexistent/part.obj\n": ("cannot read", "could not open mesh file /nonexistent/part.obj"),
    "view 0 0 1 0 0 0 60\n": ("scene has no triangles", "the config yields no triangles"),
    "mesh obj\n": ("bad mesh line", "mesh line 'obj' names no file or scene"),
}


def digest(pos, tris, tri_mat, mat_color, views) -> str:
    """One hash over the scene's float32 positions, triangles, materials,
    colours and views (float32 rows of eye, target, fov)."""
    import hashlib
    h = hashlib.sha256()
    for a, t in ((pos, np.float32), (tris, np.uint32), (tri_mat, np.uint16), (mat_color, np.float32),
                 (views, np.float32)):
        a = np.ascontiguousarray(np.asarray(a, t))
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()
