"""Facet patches of the mixed forward (lf_facet_patches, host only): every
facet lies in exactly one patch, patches stay inside one group and within 32
facets and 32 distinct corner vertices, and each patch's edge count is the
number of distinct unordered corner pairs of its facets (plus one duplicate
entry per extra pair of users of a non-manifold edge).  The kernels rely on
those bounds for their shared-memory layout."""
import ctypes as C

import numpy as np
import pytest

from lithoinv3d_b200 import _native, synth


def patches(p):
    V = np.ascontiguousarray(np.concatenate([m[0] for m in p.meshes]), np.float64)
    off = np.cumsum([0] + [len(m[0]) for m in p.meshes])
    F = np.ascontiguousarray(np.concatenate([m[1] + off[i] for i, m in enumerate(p.meshes)]), np.int32)
    go = np.cumsum([0] + [len(m[1]) for m in p.meshes]).astype(np.int32)
    lib = _native.load()
    n = C.c_int(0)
    pof = np.full(len(F), -1, np.int32)
    pv = np.zeros(len(F), np.int32)
    pe = np.zeros(len(F), np.int32)
    st = lib.lf_facet_patches(len(V), V.ctypes.data_as(_native._dp), len(F), F.ctypes.data_as(_native._ip),
                              len(go) - 1, go.ctypes.data_as(_native._ip), C.byref(n), pof.ctypes.data_as(_native._ip),
                              pv.ctypes.data_as(_native._ip), pe.ctypes.data_as(_native._ip))
    assert st == 0
    return V, F, go, n.value, pof, pv[:n.value], pe[:n.value]


@pytest.mark.parametrize("make", [lambda: synth.voxel_contact_model(shape=(12, 12, 6), n_side=4),
                                  lambda: synth.icosphere_model(subdiv=3, n_side=4),
                                  lambda: synth.batch_bodies_model(n_bodies=6, t_range=(500, 3000), side_range=(4, 6))])
def test_patch_invariants(make):
    p = make()
    V, F, go, P, pof, pv, pe = patches(p)
    assert P > 0 and np.all(pof >= 0) and np.all(pof < P)
    group = np.searchsorted(go, np.arange(len(F)), side="right") - 1
    for q in range(P):
        fs = np.nonzero(pof == q)[0]
        assert 1 <= len(fs) <= 32
        assert len(np.unique(group[fs])) == 1
        verts = np.unique(F[fs])
        assert len(verts) == pv[q] <= 32
        users = {}
        for f in fs:
            for i in range(3):
                a, b = F[f, i], F[f, (i + 1) % 3]
                key = (min(a, b), max(a, b))
                users[key] = users.get(key, 0) + 1
        assert pe[q] == sum((u + 1) // 2 for u in users.values()) <= 96
    # patches are compact: far fewer distinct vertices and edges than 3 per facet
    assert pv.sum() / len(F) < 1.0 and pe.sum() / len(F) < 2.0


def test_patch_bad_input():
    lib = _native.load()
    V = np.zeros((3, 3))
    F = np.array([[0, 1, 5]], np.int32)
    go = np.array([0, 1], np.int32)
    n = C.c_int(0)
    st = lib.lf_facet_patches(3, V.ctypes.data_as(_native._dp), 1, F.ctypes.data_as(_native._ip), 1,
                              go.ctypes.data_as(_native._ip), C.byref(n), None, None, None)
    assert st == 1
