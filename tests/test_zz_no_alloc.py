"""lf_forward_noalloc: the forward for callers that cannot allocate device
memory (a framework that owns every allocation through its own pool, a
fixed memory budget, a real-time loop).  The caller hands in device buffers;
the library uses only its built-in scratch array.  Checked against the
allocating entry point (lf_forward) on the same body, on two calls in a row
(the second call reuses the scratch the first one left behind).

This file is collected last on purpose: it must pass both alone in a fresh
process and after every other test."""
import ctypes as C

import numpy as np
import pytest

from lithoinv3d_b200 import _native, synth

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the FP64 forward tolerance used by the parity tests


def test_noalloc_forward_matches_allocating_forward():
    import torch

    lib = _native.load()
    p = synth.icosphere_model(subdiv=3, n_side=40, spacing=50.0, seed=17)
    model = p.build_model()
    ctx = p.make_context(model)
    x0 = model.assemble_parameters()
    gz_ref, tmi_ref = ctx.forward(x0)
    pos = ctx.positions(model.info().n_vertices)
    tri = model.tables()["tri"]
    ctx.close()

    dev = torch.device("cuda", 0)
    d_xyz = torch.tensor(pos, dtype=torch.float64, device=dev).contiguous()
    d_tri = torch.tensor(tri, dtype=torch.int32, device=dev).contiguous()
    d_sta = torch.tensor(p.grav_xyz, dtype=torch.float64, device=dev).contiguous()
    inc, dec, F = p.inducing
    for call in range(2):
        d_gz = torch.full((len(p.grav_xyz),), float("nan"), dtype=torch.float64, device=dev)
        d_tmi = torch.full((len(p.grav_xyz),), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        st = lib.lf_forward_noalloc(len(pos), d_xyz.data_ptr(), len(tri), d_tri.data_ptr(), len(p.grav_xyz),
                                    d_sta.data_ptr(), p.densities[0], p.susceptibilities[0], inc, dec, F,
                                    d_gz.data_ptr(), d_tmi.data_ptr(), None)
        assert st == 0, f"call {call}: status {st}"
        gz = d_gz.cpu().numpy()
        tmi = d_tmi.cpu().numpy()
        assert np.max(np.abs(gz - gz_ref)) / np.max(np.abs(gz_ref)) < TOL, call
        assert np.max(np.abs(tmi - tmi_ref)) / np.max(np.abs(tmi_ref)) < TOL, call


def test_noalloc_scratch_limited_chunking_and_single_outputs():
    """A body large enough that the facet constants leave room for fewer
    facet chunks than the launch would like (27,000 facets x 1,000 stations:
    room for 11 chunk partials against 74 wanted), so the chunk count is cut
    to fit the scratch; then each output alone (the other NULL)."""
    import torch

    lib = _native.load()
    U, F = synth.latlong_sphere(91, 150)  # 2 * 150 * 90 = 27,000 facets
    assert len(F) == 27000
    V = U * 300.0 + np.array([0.0, 0.0, -700.0])
    st = synth.station_grid(40, 40.0, 1.0, ny=25)  # 1,000 stations
    p = synth.Problem("sphere27k", [0.25], [0.03], [(V, F, synth.Z_ONLY)], st, st)
    model = p.build_model()
    ctx = p.make_context(model)
    gz_ref, tmi_ref = ctx.forward(model.assemble_parameters())
    pos = ctx.positions(model.info().n_vertices)
    tri = model.tables()["tri"]
    ctx.close()
    ns, nt = len(st), len(tri)
    doubles = 1048576 - 32 - 38 * nt
    room, want = doubles // (2 * ns), (148 * 4 + (ns + 127) // 128 - 1) // ((ns + 127) // 128)
    assert room < want, (room, want)  # the cut branch runs

    dev = torch.device("cuda", 0)
    d_xyz = torch.tensor(pos, dtype=torch.float64, device=dev).contiguous()
    d_tri = torch.tensor(tri, dtype=torch.int32, device=dev).contiguous()
    d_sta = torch.tensor(st, dtype=torch.float64, device=dev).contiguous()
    inc, dec, Fld = p.inducing

    def run(want_gz, want_tmi):
        d_gz = torch.full((ns,), float("nan"), dtype=torch.float64, device=dev)
        d_tmi = torch.full((ns,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        status = lib.lf_forward_noalloc(len(pos), d_xyz.data_ptr(), nt, d_tri.data_ptr(), ns, d_sta.data_ptr(),
                                        p.densities[0], p.susceptibilities[0], inc, dec, Fld,
                                        d_gz.data_ptr() if want_gz else None,
                                        d_tmi.data_ptr() if want_tmi else None, None)
        assert status == 0, status
        return d_gz.cpu().numpy(), d_tmi.cpu().numpy()

    gz, tmi = run(True, True)
    assert np.max(np.abs(gz - gz_ref)) / np.max(np.abs(gz_ref)) < TOL
    assert np.max(np.abs(tmi - tmi_ref)) / np.max(np.abs(tmi_ref)) < TOL
    gz_only, untouched = run(True, False)
    assert np.array_equal(gz_only, gz) and np.all(np.isnan(untouched))
    untouched, tmi_only = run(False, True)
    assert np.array_equal(tmi_only, tmi) and np.all(np.isnan(untouched))


def test_noalloc_rejects_oversize_and_bad_indices():
    import torch

    lib = _native.load()
    dev = torch.device("cuda", 0)
    xyz = torch.tensor([[0, 0, -10], [10, 0, -10], [0, 10, -10], [0, 0, -20.0]], dtype=torch.float64, device=dev)
    sta = torch.zeros((1, 3), dtype=torch.float64, device=dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    bad = torch.tensor([[0, 2, 1], [0, 1, 7]], dtype=torch.int32, device=dev)  # vertex 7 does not exist
    st = lib.lf_forward_noalloc(4, xyz.data_ptr(), 2, bad.data_ptr(), 1, sta.data_ptr(), 1.0, 0.01, 60.0, 0.0,
                                5e4, out.data_ptr(), None, None)
    assert st == 1
    # 38 * nt alone above the 8 MiB scratch: rejected before any launch
    st = lib.lf_forward_noalloc(4, xyz.data_ptr(), 40000, bad.data_ptr(), 1, sta.data_ptr(), 1.0, 0.01, 60.0, 0.0,
                                5e4, out.data_ptr(), None, None)
    assert st == 1
