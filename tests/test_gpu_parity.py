"""Parity of the CUDA path (through the C ABI) with the CPU oracle on the same seeded inputs.

Bit-exact: vertex stage, visibility (fragment list in slot order, pixel owners), neighbour
maps, image gradients, Jacobian rows and the normal equations (FP64 sums in an order shared
with the oracle). Within tolerance: the search direction (1e-4 relative to its norm) and
fitted states (1e-5 relative parameter error)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(tdi, case, synth):
    tdi.require_gpu()
    m, fr, om = case
    model = tdi.Model(m)
    batch = tdi.Batch(model, fr.n_frames)
    batch.set_frames(fr)
    lam = np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1))
    L = np.full(fr.n_frames, synth.L_INTENSITY, np.float32)
    return model, batch, lam, L


def _pose_difference(x, x_ref, K):
    """max(|tau - tau_ref|_inf / |tau_z ref|, |u - u_ref|_inf in radians): translation relative to
    the depth, rotation absolute (relative differences of near-zero components mean nothing)."""
    dt = np.abs(x[K:K + 3] - x_ref[K:K + 3]).max() / abs(float(x_ref[K + 2]))
    du = np.abs(x[K + 3:K + 6] - x_ref[K + 3:K + 6]).max()
    return float(max(dt, du))


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("case_name", ["small_case", "full_case", "rough_case"])
def test_raster_bit_exact_on_same_projections(request, tdi, synth, O, case_name):
    case = request.getfixturevalue(case_name)
    m, fr, om = case
    model, batch, lam, L = _setup(tdi, case, synth)
    for i in range(fr.n_frames):
        for state in (fr.state_true[i], fr.state_init[i]):
            geo, ok = O.vertex_stage(om, state, fr.cam[i])
            xp, yp, Z = geo[6], geo[7], geo[5]
            x0, y0 = (int(v) for v in fr.x0y0[i])
            ref = O.raster(om, xp, yp, Z, x0, y0)
            n, flags = batch.raster(i, xp, yp, Z, x0, y0)
            got = batch.read(i, tdi.READ_FRAGMENTS)
            assert n == ref["N"]
            assert np.array_equal(got["pix"], ref["pix"])
            assert np.array_equal(got["tri"], ref["tri"])
            assert np.array_equal(_bits(got["al"]), _bits(ref["al"]))
            assert np.array_equal(_bits(got["be"]), _bits(ref["be"]))
            assert np.array_equal(got["owner"], ref["owner"])


@pytest.mark.parametrize("case_name", ["small_case", "full_case", "rough_case"])
def test_evaluate_matches_oracle(request, tdi, synth, O, case_name):
    case = request.getfixturevalue(case_name)
    m, fr, om = case
    model, batch, lam, L = _setup(tdi, case, synth)
    cfg = tdi.default_config()
    ocfg = O.config()
    fs = O.FrameSet(fr)
    batch.set_state(fr.state_init, lam, L)
    batch.evaluate(cfg)
    K = m.n_expr
    for i in range(fr.n_frames):
        e = O.evaluate(om, fs, i, ocfg, fr.state_init[i], lam[i], float(L[i]))
        geo = batch.read(i, tdi.READ_GEOMETRY)
        ogeo, _ = O.vertex_stage(om, fr.state_init[i], fr.cam[i])
        for gi, oi in ((0, 0), (1, 1), (2, 2), (3, 6), (4, 7), (5, 5)):
            assert np.array_equal(_bits(geo[gi]), _bits(ogeo[oi])), ("geometry", gi)
        fr_g = batch.read(i, tdi.READ_FRAGMENTS)
        assert len(fr_g["pix"]) == e["N"]
        assert np.array_equal(fr_g["pix"], e["pix"]) and np.array_equal(fr_g["tri"], e["tri"])
        assert np.array_equal(fr_g["owner"], e["owner"])
        nb = batch.read(i, tdi.READ_NEIGHBOURS)
        assert np.array_equal(nb, e["nb"])
        gr = batch.read(i, tdi.READ_GRADIENTS)
        og = e["grads"]
        for gi, oi in ((0, 0), (1, 1), (2, 2), (3, 5), (4, 6)):
            assert np.array_equal(_bits(gr[gi]), _bits(og[oi])), ("gradient", gi)
        J = batch.read(i, tdi.READ_JACOBIAN)
        assert np.array_equal(_bits(J), _bits(e["J"]))
        ne = batch.read(i, tdi.READ_NORMAL_EQ)
        # the FP64 summation order of the normal equations is shared with the oracle
        assert np.array_equal(_bits(ne["H"]), _bits(e["H"])), np.abs(ne["H"] - e["H"]).max()
        assert np.array_equal(_bits(ne["g"]), _bits(e["g"])), np.abs(ne["g"] - e["g"]).max()
        dn = np.linalg.norm(e["d"])
        assert np.linalg.norm(ne["d"] - e["d"]) <= 1e-4 * dn
        sc = batch.read(i, tdi.READ_SCALARS)
        assert abs(sc["corr"] - e["corr"]) <= 1e-9 * abs(e["corr"])
        assert abs(sc["barrier"] - e["barrier"]) <= 1e-6 * abs(e["barrier"])
        assert abs(sc["objective"] - e["objective"]) <= 1e-6 * abs(e["objective"])
        assert sc["face_ok"] == e["face_ok"]


def test_fit_matches_oracle(tdi, synth, O, small_case):
    m, fr, om = small_case
    model, batch, lam, L = _setup(tdi, small_case, synth)
    cfg = tdi.default_config(max_iters_rigid=10)
    x, lamf, rep = batch.fit_frames(fr, fr.state_init, lam, L, cfg)
    ox, olam, orep = O.fit_frames(om, O.FrameSet(fr), O.config(max_iters_rigid=10), fr.state_init, lam, L)
    for i in range(fr.n_frames):
        assert rep[i].flags == orep[i].flags
        assert rep[i].iters_rigid == orep[i].iters_rigid
        assert rep[i].iters_lambda == orep[i].iters_lambda
        assert rep[i].n_fragments == orep[i].n_fragments
        err = np.abs(x[i] - ox[i]) / np.maximum(np.abs(ox[i]), 1e-2)
        assert err.max() <= 1e-5, err.max()
        np.testing.assert_allclose(lamf[i], olam[i], rtol=1e-5, atol=1e-7)


def test_render_skipped_frame_is_flagged_and_left_unchanged(tdi, synth, O, small_case):
    """A face too small to give 1,000 fragments: the reference skips the render
    (renderer.cu:669-677); the frame is flagged and its state stays where it started."""
    m, fr, om = small_case
    model, batch, lam, L = _setup(tdi, small_case, synth)
    x = fr.state_init.copy()
    x[0, m.n_expr + 2] *= 4.0          # four times farther away: a quarter of the size
    cfg = tdi.default_config(max_iters_rigid=5)
    xo, lamo, rep = batch.fit_frames(fr, x, lam, L, cfg)
    assert rep[0].flags & tdi.FLAG_RENDER_SKIPPED
    assert rep[0].flags & tdi.FLAG_FAIL
    assert np.array_equal(xo[0], x[0])
    assert not rep[1].flags & tdi.FLAG_RENDER_SKIPPED


def test_raster_stays_exact_across_the_depth_key_epoch_wrap(tdi, synth, O, small_case):
    """The z-buffer is never cleared between rasters: each raster's keys carry an epoch tag
    that beats all earlier ones, and the buffer is reset when the 13-bit tag range (8,191
    rasters) is used up. Rasters alternate between two poses across the reset."""
    m, fr, om = small_case
    model, batch, lam, L = _setup(tdi, small_case, synth)
    tag_max = (1 << 13) - 1
    cases = []
    for state in (fr.state_true[0], fr.state_init[0]):
        geo, ok = O.vertex_stage(om, state, fr.cam[0])
        xp, yp, Z = geo[6], geo[7], geo[5]
        x0, y0 = (int(v) for v in fr.x0y0[0])
        cases.append(((xp, yp, Z, x0, y0), O.raster(om, xp, yp, Z, x0, y0)))
    for it in range(tag_max + 4):
        args, ref = cases[it & 1]
        n, flags = batch.raster(0, *args)
        if it >= tag_max - 3:
            got = batch.read(0, tdi.READ_FRAGMENTS)
            assert n == ref["N"], it
            assert np.array_equal(got["tri"], ref["tri"]), it
            assert np.array_equal(got["owner"], ref["owner"]), it
            assert np.array_equal(got["pix"], ref["pix"]), it


@pytest.mark.parametrize("case_name", ["small_case", "full_case"])
def test_tensor_core_normal_equations_within_fp32_accumulation_error(request, tdi, synth, O, case_name):
    """normal_eq = 1: J^T J and J^T r from split-BF16 products on the tensor cores, FP32
    accumulation per 256-fragment chunk. Against the oracle's FP64 sums: relative error of H
    (Frobenius) and of g (max norm) within 1e-5, the class of the reference's own cublasSgemm."""
    case = request.getfixturevalue(case_name)
    m, fr, om = case
    model, batch, lam, L = _setup(tdi, case, synth)
    cfg = tdi.default_config(normal_eq=tdi.NORMAL_EQ_TENSOR)
    fs = O.FrameSet(fr)
    batch.set_state(fr.state_init, lam, L)
    batch.evaluate(cfg)
    for i in range(fr.n_frames):
        e = O.evaluate(om, fs, i, O.config(), fr.state_init[i], lam[i], float(L[i]))
        ne = batch.read(i, tdi.READ_NORMAL_EQ)
        H, Ho = ne["H"].astype(np.float64), e["H"].astype(np.float64)
        assert np.array_equal(H, H.T)
        assert np.linalg.norm(H - Ho) <= 1e-5 * np.linalg.norm(Ho)
        assert np.abs(ne["g"] - e["g"]).max() <= 1e-5 * np.abs(e["g"]).max()
        # everything upstream of the normal equations is unchanged
        assert np.array_equal(_bits(batch.read(i, tdi.READ_JACOBIAN)), _bits(e["J"]))


def test_tensor_core_fit_reaches_the_exact_fits_objective(tdi, synth, O, small_case):
    """Fits with tensor-core normal equations follow different (rounding-level) search
    directions, so their iterates are not the oracle's; they must end at an objective within
    0.5% of the exact fit's, with the same status flags (apart from TDI_FLAG_FAIL, which marks a
    shape fit of at most NITERS_SUCCESS outer iterations: a count the two can land on either
    side of), and with the pose (the well-determined parameters) close to the exact fit's: the
    larger of the translation difference relative to the depth and the rotation-vector difference
    in radians at most 1e-2 (median over frames; 5e-2 at most)."""
    m, fr, om = small_case
    model, batch, lam, L = _setup(tdi, small_case, synth)
    x0, lam0, rep0 = batch.fit_frames(fr, fr.state_init, lam, L, tdi.default_config(max_iters_rigid=10))
    x1, lam1, rep1 = batch.fit_frames(fr, fr.state_init, lam, L,
                                      tdi.default_config(max_iters_rigid=10, normal_eq=tdi.NORMAL_EQ_TENSOR))
    K = m.n_expr
    pose_err = []
    for i in range(fr.n_frames):
        assert (rep1[i].flags | tdi.FLAG_FAIL) == (rep0[i].flags | tdi.FLAG_FAIL)
        assert abs(rep1[i].objective - rep0[i].objective) <= 5e-3 * abs(rep0[i].objective)
        # pose (translation and rotation), the well-determined group, at parameter level
        pose_err.append(_pose_difference(x1[i], x0[i], K))
    print("tensor vs exact fit, pose relative difference per frame:", pose_err)
    assert np.median(pose_err) <= 1e-2 and max(pose_err) <= 5e-2


@pytest.mark.parametrize("case_name", ["small_case", "full_case"])
def test_graph_rounds_equal_host_rounds(request, tdi, synth, O, case_name):
    """Stage rounds replayed from CUDA graphs (the default: kernels read the active-frame count
    from device memory, the host reads it once per 16 rounds) give the fits of host-driven
    rounds bit for bit, including the two-stage illumination and the finetune."""
    case = request.getfixturevalue(case_name)
    m, fr, om = case
    model, batch, lam, L = _setup(tdi, case, synth)
    kw = dict(max_iters_rigid=10, max_iters_finetune=10, twostage_illum=1, finetune=1)
    n0 = batch.launches()
    xg, lg, rg = batch.fit_frames(fr, fr.state_init, lam, L, tdi.default_config(**kw))
    n1 = batch.launches()
    xh, lh, rh = batch.fit_frames(fr, fr.state_init, lam, L, tdi.default_config(host_rounds=1, **kw))
    assert np.array_equal(xg.view(np.uint32), xh.view(np.uint32))
    assert np.array_equal(lg.view(np.uint32), lh.view(np.uint32))
    for a, b in zip(rg, rh):
        assert (a.flags, a.iters_rigid, a.iters_finetune, a.iters_lambda, a.renders) == \
               (b.flags, b.iters_rigid, b.iters_finetune, b.iters_lambda, b.renders)
    assert n1 > n0
