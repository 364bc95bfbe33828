"""The allocation-free visibility entry point (tdi_raster_noalloc) against the batch one.

tdi_raster_noalloc serves callers that may not allocate device memory (a plugin in an
application that owns the device pool, a fixed memory budget): its working memory is a fixed
array inside the library. Its fragments must equal tdi_batch_raster's for the same
projections, on consecutive calls (the second call must not see the first one's depth keys).
This file is collected last; it runs alone or after the other tests.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _project(m, fr, i, state):
    """Projected vertices of frame i at a state (float64, rounded to float32)."""
    synth = importlib.import_module("3di_b200.synth")
    K = m.n_expr
    R = synth.rodrigues(state[K + 3:].astype(np.float64))
    P = m.mean.astype(np.float64) + np.einsum("vck,k->cv", m.E.astype(np.float64), state[:K].astype(np.float64))
    Pc = R @ P + state[K:K + 3, None].astype(np.float64)
    phix, phiy, cx, cy = fr.cam[i].astype(np.float64)
    xp = (phix * Pc[0] / Pc[2] + cx).astype(np.float32)
    yp = (phiy * Pc[1] / Pc[2] + cy).astype(np.float32)
    return xp, yp, Pc[2].astype(np.float32)


def test_noalloc_raster_equals_batch_raster_on_consecutive_calls():
    tdi = importlib.import_module("3di_b200")
    synth = importlib.import_module("3di_b200.synth")
    tdi.require_gpu()
    import torch
    m = synth.make_model(5000, 9800, 0)
    fr = synth.make_frames(m, 2, 0)
    model = tdi.Model(m)
    batch = tdi.Batch(model, 1)
    lib = tdi.load_library()
    dev = torch.device("cuda", 0)
    tl = torch.from_numpy(np.ascontiguousarray(m.tl, dtype=np.int32)).to(dev)
    cap = 4 * m.n_triangles
    out = torch.full((cap * 4,), -7, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    for i, state in ((0, fr.state_true[0]), (1, fr.state_init[1])):
        xp, yp, zc = _project(m, fr, i, state)
        x0, y0 = (int(v) for v in fr.x0y0[i])
        n_ref, flags_ref = batch.raster(0, xp, yp, zc, x0, y0)
        ref = batch.read(0, tdi.READ_FRAGMENTS)
        d = [torch.from_numpy(a).to(dev) for a in (xp, yp, zc)]
        st = lib.tdi_raster_noalloc(C.c_void_p(d[0].data_ptr()), C.c_void_p(d[1].data_ptr()),
                                    C.c_void_p(d[2].data_ptr()), C.c_void_p(tl.data_ptr()),
                                    m.n_vertices, m.n_triangles, x0, y0, C.c_void_p(out.data_ptr()),
                                    cap, C.c_void_p(count.data_ptr()), C.c_void_p(flags.data_ptr()), None)
        assert st == 0, lib.tdi_last_error()
        torch.cuda.synchronize()
        n = int(count.item())
        assert n == n_ref and n > 1000
        assert int(flags.item()) & 0xFFFFFFFF == flags_ref
        got = out[:4 * n].cpu().numpy().reshape(n, 4)
        po = got[:, 0].view(np.uint32)
        assert np.array_equal((po & 0xFFFF).astype(np.uint16), ref["pix"])
        assert np.array_equal((po >> 31).astype(np.uint8), ref["owner"])
        assert np.array_equal(got[:, 1], ref["tri"])
        assert np.array_equal(got[:, 2].view(np.float32).view(np.uint32), ref["al"].view(np.uint32))
        assert np.array_equal(got[:, 3].view(np.float32).view(np.uint32), ref["be"].view(np.uint32))


def _noalloc(lib, dev_arrays, tl, V, T, x0, y0, out, cap, count, flags):
    d = dev_arrays
    return lib.tdi_raster_noalloc(C.c_void_p(d[0].data_ptr()), C.c_void_p(d[1].data_ptr()),
                                  C.c_void_p(d[2].data_ptr()), C.c_void_p(tl.data_ptr()), V, T, x0, y0,
                                  C.c_void_p(out.data_ptr()), cap, C.c_void_p(count.data_ptr()),
                                  C.c_void_p(flags.data_ptr()), None)


def test_noalloc_raster_overflow_stops_at_capacity():
    """With room for half of the fragments the count stops at capacity, the overflow flag is
    set, the records written are the first ones of the full list and nothing is written past
    capacity (a guard region of sentinels after it stays unchanged)."""
    tdi = importlib.import_module("3di_b200")
    synth = importlib.import_module("3di_b200.synth")
    tdi.require_gpu()
    import torch
    m = synth.make_model(5000, 9800, 0)
    fr = synth.make_frames(m, 1, 0)
    model = tdi.Model(m)
    batch = tdi.Batch(model, 1)
    lib = tdi.load_library()
    dev = torch.device("cuda", 0)
    tl = torch.from_numpy(np.ascontiguousarray(m.tl, dtype=np.int32)).to(dev)
    xp, yp, zc = _project(m, fr, 0, fr.state_true[0])
    x0, y0 = (int(v) for v in fr.x0y0[0])
    n_ref, flags_ref = batch.raster(0, xp, yp, zc, x0, y0)
    ref = batch.read(0, tdi.READ_FRAGMENTS)
    cap, guard = n_ref // 2, 1024
    out = torch.full(((cap + guard) * 4,), -7, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    d = [torch.from_numpy(a).to(dev) for a in (xp, yp, zc)]
    st = _noalloc(lib, d, tl, m.n_vertices, m.n_triangles, x0, y0, out, cap, count, flags)
    assert st == 0, lib.tdi_last_error()
    torch.cuda.synchronize()
    assert int(count.item()) == cap
    assert int(flags.item()) & tdi.FLAG_OVERFLOW
    got = out.cpu().numpy()
    assert np.all(got[4 * cap:] == -7), "records written past capacity"
    rec = got[:4 * cap].reshape(cap, 4)
    assert np.array_equal(rec[:, 1], ref["tri"][:cap])
    assert np.array_equal((rec[:, 0].view(np.uint32) & 0xFFFF).astype(np.uint16), ref["pix"][:cap])


def test_noalloc_raster_skips_triangles_with_a_corner_outside_the_vertices():
    """A corner index equal to n_vertices: the triangle is skipped before any vertex read and
    the call reports TDI_FLAG_BAD_INDEX. The vertex arrays are padded, so that even an
    unchecked read would stay inside the allocation."""
    tdi = importlib.import_module("3di_b200")
    synth = importlib.import_module("3di_b200.synth")
    tdi.require_gpu()
    import torch
    m = synth.make_model(5000, 9800, 0)
    fr = synth.make_frames(m, 1, 0)
    lib = tdi.load_library()
    dev = torch.device("cuda", 0)
    xp, yp, zc = _project(m, fr, 0, fr.state_true[0])
    x0, y0 = (int(v) for v in fr.x0y0[0])
    V, T = m.n_vertices, m.n_triangles
    pad = 64
    d = [torch.from_numpy(np.concatenate([a, np.full(pad, a.mean(), np.float32)])).to(dev) for a in (xp, yp, zc)]
    tl_h = np.ascontiguousarray(m.tl, dtype=np.int32).copy()
    cap = 4 * T
    out = torch.full((cap * 4,), -7, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    tl = torch.from_numpy(tl_h).to(dev)
    assert _noalloc(lib, d, tl, V, T, x0, y0, out, cap, count, flags) == 0, lib.tdi_last_error()
    torch.cuda.synchronize()
    n0 = int(count.item())
    tris0 = out[:4 * n0].cpu().numpy().reshape(n0, 4)[:, 1]
    assert not int(flags.item()) & tdi.FLAG_BAD_INDEX
    bad = int(tris0[n0 // 2])                   # a triangle that has fragments
    tl_h[0, bad] = V
    tl = torch.from_numpy(tl_h).to(dev)
    assert _noalloc(lib, d, tl, V, T, x0, y0, out, cap, count, flags) == 0, lib.tdi_last_error()
    torch.cuda.synchronize()
    n1 = int(count.item())
    tris1 = out[:4 * n1].cpu().numpy().reshape(n1, 4)[:, 1]
    assert int(flags.item()) & tdi.FLAG_BAD_INDEX
    assert bad not in set(tris1.tolist())
    assert n1 > 1000


def test_noalloc_raster_rejects_meshes_above_its_fixed_size():
    tdi = importlib.import_module("3di_b200")
    tdi.require_gpu()
    lib = tdi.load_library()
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    st = lib.tdi_raster_noalloc(dummy, dummy, dummy, dummy, 10, 131073, 0, 0, dummy, 16, dummy, dummy, None)
    assert st == 4 and b"131072" in lib.tdi_last_error()


def test_noalloc_raster_equals_oracle_on_the_full_size_mesh(O, full_case):
    """The 53,490-vertex / 106,466-triangle mesh (the size the fixed 131,072-triangle working
    array is for), at the true and the initial states of each frame: fragments bit for bit the
    oracle's (count, slot order, pixels, triangles, barycentric bits, owners)."""
    tdi = importlib.import_module("3di_b200")
    tdi.require_gpu()
    import torch
    m, fr, om = full_case
    lib = tdi.load_library()
    dev = torch.device("cuda", 0)
    tl = torch.from_numpy(np.ascontiguousarray(m.tl, dtype=np.int32)).to(dev)
    cap = 4 * m.n_triangles
    out = torch.zeros(cap * 4, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    for i in range(fr.n_frames):
        for state in (fr.state_true[i], fr.state_init[i]):
            geo, ok = O.vertex_stage(om, state, fr.cam[i])
            xp, yp, zc = geo[6], geo[7], geo[5]
            x0, y0 = (int(v) for v in fr.x0y0[i])
            ref = O.raster(om, xp, yp, zc, x0, y0)
            d = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev) for a in (xp, yp, zc)]
            st = _noalloc(lib, d, tl, m.n_vertices, m.n_triangles, x0, y0, out, cap, count, flags)
            assert st == 0, lib.tdi_last_error()
            torch.cuda.synchronize()
            n = int(count.item())
            assert n == ref["N"] and n > 1000
            got = out[:4 * n].cpu().numpy().reshape(n, 4)
            po = got[:, 0].view(np.uint32)
            assert np.array_equal((po & 0xFFFF).astype(np.uint16), ref["pix"])
            assert np.array_equal((po >> 31).astype(np.uint8), ref["owner"])
            assert np.array_equal(got[:, 1], ref["tri"])
            assert np.array_equal(got[:, 2].view(np.uint32), ref["al"].view(np.uint32))
            assert np.array_equal(got[:, 3].view(np.uint32), ref["be"].view(np.uint32))
