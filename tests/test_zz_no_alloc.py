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


def test_noalloc_raster_rejects_meshes_above_its_fixed_size():
    tdi = importlib.import_module("3di_b200")
    tdi.require_gpu()
    lib = tdi.load_library()
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    st = lib.tdi_raster_noalloc(dummy, dummy, dummy, dummy, 10, 131073, 0, 0, dummy, 16, dummy, dummy, None)
    assert st == 4 and b"131072" in lib.tdi_last_error()
