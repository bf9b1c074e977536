"""CPU: the METIS ordering of the CEMAS banks, regenerated from the unsorted meshes.

The reference orders a mesh for its 16-vertex MAS banks offline
(MeshProcess/metis_partition/src/metis_sort.cpp): METIS k-way partitions of the vertex graph
with nPart = ceil(V / (16 - s)), s raised until no part exceeds 16 vertices, then the
vertices are sorted by part.  It ships the results for four meshes as
Assets/sorted_mesh/*_sorted.16.{msh,obj,part} (tests/golden/*_sorted16.npz).  Here METIS and
GKlib are compiled from the reference's own vendored C sources (oracle/Makefile `ref`) and
driven by oracle/metis_sort.cpp; the shipped files were made by a Windows build, so METIS's
rand() is the Microsoft runtime's (oracle/crt_rand.c).

Bars, per mesh: the sorted part sequence (the .part file) bit-exact, the same slack s and
part count, and every part holding the same vertices (matched by position) as the shipped
sorted mesh.  The order of the vertices inside a part is std::sort's (not stable), which
differs between the Microsoft and GNU standard libraries, so it is not compared.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

LIB = os.path.join(ROOT, "oracle", "_ref", "libstg_metis.so")

pytestmark = pytest.mark.skipif(not os.path.exists(LIB),
                                reason="oracle/_ref/libstg_metis.so not built (make -C oracle ref needs the "
                                       "reference's METIS sources)")


def _metis_sort(elems, nv, bank=16):
    L = C.CDLL(LIB)
    L.orc_metis_sort.restype = C.c_int
    el = np.ascontiguousarray(elems, np.int32)
    part = np.zeros(nv, np.int32)
    order = np.zeros(nv, np.int32)
    slack = C.c_int()
    npart = L.orc_metis_sort(nv, el.shape[0], el.shape[1], el.ctypes.data_as(C.c_void_p), bank,
                             part.ctypes.data_as(C.c_void_p), order.ctypes.data_as(C.c_void_p), C.byref(slack))
    return npart, part, order, slack.value


# (mesh, parts, slack): nPart = (V + 16 - s - 1) // (16 - s) at the slack the shipped files need
CASES = [("cube", 1, 0), ("cloth_high", 282, 1), ("bunny2", 1280, 1), ("high_mat", 3000, 1)]


@pytest.mark.parametrize("name,parts,slack", CASES)
def test_metis_regenerates_shipped_partition(name, parts, slack):
    src = np.load(os.path.join(GOLDEN, f"{name}_input.npz"))
    ref = np.load(os.path.join(GOLDEN, f"{name}_sorted16.npz"))
    pos, elems = src["pos"], src["elems"]
    nv = pos.shape[0]
    npart, part, order, s = _metis_sort(elems, nv)
    assert (npart, s) == (parts, slack)
    assert np.bincount(part, minlength=npart).max() <= 16
    # the .part file: the part of every vertex of the sorted mesh
    shipped = ref["part"]
    assert np.array_equal(part[order], shipped)
    # every part holds the shipped part's vertices (float32 positions, sorted per part)
    sp, P, Q = part[order], pos[order], ref["pos"]
    for p in range(npart):
        a, b = P[sp == p], Q[shipped == p]
        a = a[np.lexsort(a.T[::-1])]
        b = b[np.lexsort(b.T[::-1])]
        assert a.shape == b.shape and np.allclose(a, b, rtol=1e-6, atol=1e-6), (name, p)


def test_metis_order_is_a_permutation_grouped_by_part():
    src = np.load(os.path.join(GOLDEN, "bunny2_input.npz"))
    nv = src["pos"].shape[0]
    _, part, order, _ = _metis_sort(src["elems"], nv)
    assert np.array_equal(np.sort(order), np.arange(nv))
    assert np.all(np.diff(part[order]) >= 0)


def test_metis_rejects_bad_input():
    assert _metis_sort(np.array([[0, 1, 2, 9]], np.int32), 4)[0] == -1   # vertex id out of range
