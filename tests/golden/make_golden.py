"""Regenerate the golden fixtures from the reference's shipped assets.

    python tests/golden/make_golden.py <reference checkout>

The reference checkout is the first argument, or the STG_REFERENCE_ROOT environment
variable.  Reads Assets/sorted_mesh/{cube,bunny2,high_mat}_sorted.16.{msh,part} and
cloth_high_sorted.16.{obj,part}
(the METIS-partitioned, partition-sorted meshes the reference ships; produced by
MeshProcess/metis_partition/src/metis_sort.cpp) and stores their element connectivity,
vertex positions and per-vertex partition ids as compressed .npz files next to this script.
These pin the CEMAS ordering inputs (partId per vertex, vertices grouped by part) for the
MAS hierarchy tests.  The unsorted meshes they were made from (Assets/tetMesh/{cube,bunny2,
high_mat}.msh, Assets/triMesh/cloth_high.obj) are stored as *_input.npz (positions, elements)
for the METIS regeneration test (tests/test_metis_cpu.py); nothing else is taken from the
reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_msh(path):
    """gmsh 2.2 ASCII as the reference's TetMesh loader reads it (MeshProcess/metis_partition/
    src/mesh.cpp:265-335): a node is the last three fields of its line, an element the last
    four (Assets/tetMesh/bunny2.msh declares two tags per element but writes none)."""
    with open(path) as f:
        lines = f.read().split("\n")
    i = lines.index("$Nodes")
    nn = int(lines[i + 1])
    pos = np.array([[float(t) for t in lines[i + 2 + k].split()[-3:]] for k in range(nn)])
    j = lines.index("$Elements")
    ne = int(lines[j + 1])
    tets = [[int(v) - 1 for v in lines[j + 2 + k].split()[-4:]] for k in range(ne)]
    return pos, np.array(tets, dtype=np.int32)


def read_obj(path):
    pos, tris = [], []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                pos.append([float(a) for a in t[1:4]])
            elif t[0] == "f":
                tris.append([int(a.split("/")[0]) - 1 for a in t[1:4]])
    return np.array(pos), np.array(tris, dtype=np.int32)


def read_part(path):
    return np.loadtxt(path, dtype=np.int32).reshape(-1)


def main(ref_root):
    sm = os.path.join(ref_root, "Assets", "sorted_mesh")
    for name in ("cube", "bunny2", "high_mat"):
        pos, tets = read_msh(os.path.join(sm, f"{name}_sorted.16.msh"))
        part = read_part(os.path.join(sm, f"{name}_sorted.16.part"))
        assert part.size == pos.shape[0], (name, part.size, pos.shape)
        np.savez_compressed(os.path.join(HERE, f"{name}_sorted16.npz"), pos=pos.astype(np.float32), tets=tets, part=part)
        print(name, pos.shape[0], "verts", tets.shape[0], "tets")
    pos, tris = read_obj(os.path.join(sm, "cloth_high_sorted.16.obj"))
    part = read_part(os.path.join(sm, "cloth_high_sorted.16.part"))
    assert part.size == pos.shape[0]
    np.savez_compressed(os.path.join(HERE, "cloth_high_sorted16.npz"), pos=pos.astype(np.float32), tris=tris, part=part)
    print("cloth_high", pos.shape[0], "verts", tris.shape[0], "tris")
    # the unsorted meshes the METIS ordering starts from (Assets/tetMesh, Assets/triMesh)
    for name in ("cube", "bunny2", "high_mat"):
        pos, tets = read_msh(os.path.join(ref_root, "Assets", "tetMesh", f"{name}.msh"))
        np.savez_compressed(os.path.join(HERE, f"{name}_input.npz"), pos=pos.astype(np.float32), elems=tets)
    pos, tris = read_obj(os.path.join(ref_root, "Assets", "triMesh", "cloth_high.obj"))
    np.savez_compressed(os.path.join(HERE, "cloth_high_input.npz"), pos=pos.astype(np.float32), elems=tris)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("STG_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout>  (or set STG_REFERENCE_ROOT)")
    main(root)
