"""Surface files (lf_read_surface, lf_write_tsurf) against the reference's
own loaders and TSurf exporter (oracle/_ref: loadSurfaceMesh,
InversionExporter::exportTS): identical vertices (same doubles), triangles
and written text on hand-made files that exercise every rule of the
readers, and -- where the reference tree is present -- on the real
Forrestania group meshes.  CPU only (no device code involved)."""
import glob
import os

import numpy as np
import pytest

from oracle_bindings import ref_available, ref_export_ts, ref_load_surface
from lithoinv3d_b200 import LithoError, read_surface, synth, write_tsurf

needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")

TS_TEXT = """GOCAD TSurf 1
HEADER {
name:odd_one
 VRTX 99 1 2 3
}
# a comment
   TFACE
VRTX 1 10.5 -3.25e2 7
PVRTX 2 0.1 0.2 0.3 4.5
VRTX 3 -1 -2 -3
VRTX 4 1.0000000001 2 3
VRTX 5 bad line
TRIANGLES
TRGL 1 2 3
TRGL 2 3 4
TRGL 1 2
END
VRTX 6 9 9 9
"""

OBJ_TEXT = """# comment
v 0 0 0
v 1 0 0
  v 1 1 0
v 0 1 0
v 0.5 0.5 1.25
vn 0 0 1
f 1/1/1 2/2/1 3/3/1 4/4/1
fo 1 2 5
f 3 x 5
f 1 2
"""


def write(path, text, crlf=False):
    with open(path, "w", newline="") as fh:
        fh.write(text.replace("\n", "\r\n") if crlf else text)


@needs_ref
@pytest.mark.parametrize("crlf", [False, True])
def test_reader_matches_reference_on_crafted_files(tmp_path, crlf):
    for name, text in (("a.ts", TS_TEXT), ("b.obj", OBJ_TEXT)):
        path = tmp_path / name
        write(path, text, crlf)
        want = ref_load_surface(path)
        assert want is not None
        xyz, tri = read_surface(path)
        assert np.array_equal(xyz, want[0]) and np.array_equal(tri, want[1])
    # the TSurf rules: header skipped, malformed vertex and triangle lines
    # skipped, END stops (LF endings; with CRLF the END line keeps its '\r')
    xyz, tri = read_surface(tmp_path / "a.ts")
    if not crlf:
        assert len(xyz) == 4 and tri.tolist() == [[0, 1, 2], [1, 2, 3]]
    # the OBJ rules: quad fanned, "fo" accepted, bad and short faces skipped
    xyz, tri = read_surface(tmp_path / "b.obj")
    assert tri.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 4]]


@needs_ref
def test_writer_matches_reference_exporter(tmp_path):
    p = synth.voxel_contact_model(shape=(4, 4, 3), n_side=4, cp_stride=0)
    V, F, _ = p.meshes[1]
    V = np.asarray(V) + np.random.default_rng(0).normal(0, 1e-3, np.shape(V))
    ref_export_ts(tmp_path, "model", "group1", V, F)
    write_tsurf(tmp_path / "ours.ts", "model_group1", V, F)
    assert (tmp_path / "ours.ts").read_text() == (tmp_path / "model_group1.ts").read_text()
    xyz, tri = read_surface(tmp_path / "ours.ts")
    assert np.allclose(xyz, V, rtol=1e-8, atol=1e-6) and np.array_equal(tri, np.asarray(F))


@needs_ref
def test_reader_on_real_group_meshes():
    root = os.environ.get("LITHO_REFERENCE")
    if not root:
        pytest.skip("LITHO_REFERENCE (the reference tree) is not set")
    files = sorted(glob.glob(os.path.join(root, "apps/forrestania/*/baseline/meshes/volume_group_*.ts")))
    if not files:
        pytest.skip("reference meshes not present")
    total = 0
    for f in files:
        want = ref_load_surface(f)
        xyz, tri = read_surface(f)
        assert np.array_equal(xyz, want[0]) and np.array_equal(tri, want[1])
        total += len(tri)
    assert total > 10000


def test_reader_errors(tmp_path):
    with pytest.raises(LithoError):
        read_surface(tmp_path / "missing.ts")
    write(tmp_path / "x.stl", "solid\n")
    with pytest.raises(LithoError):
        read_surface(tmp_path / "x.stl")
    write(tmp_path / "empty.ts", "GOCAD TSurf 1\nTFACE\nEND\n")
    with pytest.raises(LithoError):
        read_surface(tmp_path / "empty.ts")
    write(tmp_path / "range.obj", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n")
    with pytest.raises(LithoError):  # the reference would return this mesh unchecked
        read_surface(tmp_path / "range.obj")
    with pytest.raises(LithoError):
        write_tsurf(tmp_path / "w.ts", "w", np.zeros((3, 3)), [[0, 1, 3]])
