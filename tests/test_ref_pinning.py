"""The oracle pinned to 3DI itself: the reference's own CUDA kernels, compiled unmodified from
its sources into oracle/_ref/ (oracle/ref.mk), run on the same inputs as the oracle and the
product, stage by stage.

Each stage gets identical inputs on both sides (the oracle's projections for the raster, its
geometry and rotation for the evaluation), so that a difference points at one stage. With the
reference built without FMA contraction (the oracle's arithmetic contract) every elementwise
output is compared bit for bit; with nvcc's default flags (how the reference's own CMake
build compiles it) the mismatch counts are reported and bounded. The reference forms J^T J,
J^T r and the correlation with cuBLAS (derivative_computer.cu:157-164, renderer.cu:725-729),
whose summation order is the library's: those are compared within FP32 accumulation error.

Known reference behaviours that this build does not reproduce, shown here:
* pixels covered by several fragments of equal depth are painted by whichever thread writes
  last (funcs.cu:816); the oracle and the product paint the lowest triangle id. Stages that
  read the painted image are compared away from such pixels;
* the Renderer never resets its slot buffers between renders (renderer.cu:64-68 allocate
  them once; keep_only_minZ scans all slots, funcs.cu:1016-1029), so a slot left over from
  an earlier render survives when its old depth equals the pixel's new minimum.
"""
import importlib

import numpy as np
import pytest

import refpin
from conftest import make_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_reference():
    tdi = importlib.import_module("3di_b200")
    tdi.require_gpu()
    if not refpin.available():
        pytest.skip("oracle/_ref/ not built (needs the 3DI sources; make -f oracle/ref.mk)")


@pytest.fixture(scope="module")
def ref_size_case(synth, O):
    """19,830 vertices / 39,053 triangles: the size of the model 3DI ships with
    (BFMmm-19830), within its 16-bit indices; 1080p frames rescaled to the crop."""
    return make_case(synth, O, 19830, 39053, 2, 2, dict(image_wh=(1920, 1080), box_range=(300, 600)))


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _states(fr):
    return [(i, s) for i in range(fr.n_frames) for s in (fr.state_true[i], fr.state_init[i])]


def test_rotation_within_two_units_in_the_last_place(synth, O, small_case):
    """fill_theta_etc (rotation_header.cu:46-151) evaluates sinf/cosf in FP32; the oracle and
    the product evaluate sin/cos in FP64 and round (the one intentional difference in the
    rotation). R and dR agree to within 2 units in the last place of 1."""
    m, fr, om = small_case
    rs = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75])
    K = m.n_expr
    same = total = 0
    for i, s in _states(fr):
        R, dR = rs.rotation(s[K + 3:])
        Ro, dRo = O.rotation(s[K + 3:])
        ulp = np.spacing(np.float32(1.0))
        assert np.abs(R - Ro).max() <= 2 * ulp
        assert np.abs(dR - dRo).max() <= 2 * ulp * max(1.0, np.abs(dRo).max())
        same += int(np.sum(_bits(R) == _bits(Ro))) + int(np.sum(_bits(dR) == _bits(dRo)))
        total += R.size + dR.size
    print(f"rotation: {same}/{total} entries bit-equal to the reference")


@pytest.mark.parametrize("nofma", [True, False])
def test_view_transform_matches_reference(synth, O, small_case, nofma):
    """view_transform_3d_pts_and_render_2d (funcs.cu:395-453) on the oracle's object points and
    rotation: bit-equal without FMA contraction; with nvcc's default contraction the
    projections differ in the last bits only."""
    m, fr, om = small_case
    rs = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75], nofma=nofma)
    K = m.n_expr
    for i, s in _states(fr):
        geo, _ = O.vertex_stage(om, s, fr.cam[i])
        R, _ = O.rotation(s[K + 3:])
        out = rs.view_transform(geo[0], geo[1], geo[2], R, s[K:K + 3], fr.cam[i])
        for q, g in enumerate((3, 4, 5, 6, 7)):
            if nofma:
                assert np.array_equal(_bits(out[q]), _bits(geo[g])), q
            else:
                np.testing.assert_allclose(out[q], geo[g], rtol=1e-5, atol=1e-5)


def _raster_cases(request, O, case_name):
    case = request.getfixturevalue(case_name)
    m, fr, om = case
    out = []
    for i, s in _states(fr):
        geo, _ = O.vertex_stage(om, s, fr.cam[i])
        out.append((geo[6], geo[7], geo[5], int(fr.x0y0[i, 0]), int(fr.x0y0[i, 1])))
    return case, out


@pytest.mark.parametrize("case_name", ["small_case", "ref_size_case"])
def test_raster_bit_exact_against_reference(request, tdi, synth, O, case_name):
    """get_pixels_to_render, keep_only_minZ and remove_if (funcs.cu:915-1029,
    renderer.cu:640-677) against the oracle's raster and the product's, on fresh reference
    buffers: survivor count, slot order, pixels, triangles and barycentric bits."""
    (m, fr, om), cases = _raster_cases(request, O, case_name)
    model = tdi.Model(m)
    batch = tdi.Batch(model, 1)
    for xp, yp, Z, x0, y0 in cases:
        rs = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75], nofma=True)
        ref = rs.raster(xp, yp, Z, x0, y0)
        rs.close()
        o = O.raster(om, xp, yp, Z, x0, y0)
        assert ref["N"] == o["N"]
        assert np.array_equal(ref["pix"], o["pix"]) and np.array_equal(ref["tri"], o["tri"])
        assert np.array_equal(_bits(ref["al"]), _bits(o["al"]))
        assert np.array_equal(_bits(ref["be"]), _bits(o["be"]))
        n, _ = batch.raster(0, xp, yp, Z, x0, y0)
        got = batch.read(0, tdi.READ_FRAGMENTS)
        assert n == ref["N"]
        assert np.array_equal(got["pix"], ref["pix"]) and np.array_equal(got["tri"], ref["tri"])
        assert np.array_equal(_bits(got["al"]), _bits(ref["al"]))


@pytest.mark.parametrize("case_name", ["small_case", "ref_size_case"])
def test_raster_against_reference_built_with_contraction(request, synth, O, case_name):
    """The reference as its CMake build compiles it (nvcc's default FMA contraction): the
    barycentrics differ in the last bits and points on a triangle's edge can flip; the visible
    set stays within 0.5% of the uncontracted one."""
    (m, fr, om), cases = _raster_cases(request, O, case_name)
    for xp, yp, Z, x0, y0 in cases:
        rs = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75], nofma=False)
        ref = rs.raster(xp, yp, Z, x0, y0)
        rs.close()
        o = O.raster(om, xp, yp, Z, x0, y0)
        a = set(zip(ref["pix"].tolist(), ref["tri"].tolist()))
        b = set(zip(o["pix"].tolist(), o["tri"].tolist()))
        diff = len(a ^ b)
        print(f"contracted build: N {ref['N']} vs {o['N']}, {diff} fragments differ")
        assert diff <= 0.005 * o["N"]


def test_reference_keeps_stale_slots_across_renders(synth, O, small_case):
    """Two renders in a row on the same reference buffers, the second with only tau_x moved
    (camera depths unchanged, projections shifted by a fraction of a pixel). Slots the second
    render no longer writes keep their first-render pixel and depth, and survive where that
    depth equals the pixel's new minimum: the reference's list is the fresh one plus such
    leftovers. This build renders from fresh state (a departure that makes each render depend
    only on its own inputs)."""
    m, fr, om = small_case
    K = m.n_expr
    s_a = fr.state_true[0].copy()
    s_b = s_a.copy()
    s_b[K] += np.float32(0.37 * s_a[K + 2] / fr.cam[0][0])   # ~0.37 px in x
    ga, _ = O.vertex_stage(om, s_a, fr.cam[0])
    gb, _ = O.vertex_stage(om, s_b, fr.cam[0])
    assert np.array_equal(_bits(ga[5]), _bits(gb[5]))          # depths unchanged
    x0, y0 = (int(v) for v in fr.x0y0[0])
    seq = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75], nofma=True)
    ra = seq.raster(ga[6], ga[7], ga[5], x0, y0)
    rb_seq = seq.raster(gb[6], gb[7], gb[5], x0, y0)
    fresh = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75], nofma=True)
    rb = fresh.raster(gb[6], gb[7], gb[5], x0, y0)
    ob = O.raster(om, gb[6], gb[7], gb[5], x0, y0)
    assert rb["N"] == ob["N"] and np.array_equal(rb["tri"], ob["tri"])
    seq_set = list(zip(rb_seq["pix"].tolist(), rb_seq["tri"].tolist()))
    fresh_set = set(zip(rb["pix"].tolist(), rb["tri"].tolist()))
    a_set = set(zip(ra["pix"].tolist(), ra["tri"].tolist()))
    extra = [f for f in seq_set if f not in fresh_set]
    assert fresh_set <= set(seq_set)
    assert all(f in a_set for f in extra)        # every extra fragment is a first-render leftover
    print(f"stale survivors: {len(extra)} of {rb_seq['N']}")
    assert len(extra) > 0


def _race_pixels(o):
    """Pixels with several survivors whose shaded values differ: the reference's painter races
    there (funcs.cu:816)."""
    pix = o["pix"].astype(np.int64)
    shade = _bits(o["sh"][0])
    order = np.argsort(pix, kind="stable")
    ps, ss = pix[order], shade[order]
    race = set()
    start = 0
    for k in range(1, len(ps) + 1):
        if k == len(ps) or ps[k] != ps[start]:
            if k - start > 1 and len(set(ss[start:k].tolist())) > 1:
                race.add(int(ps[start]))
            start = k
    return race


def _far_from(pix, race, r):
    """Mask of fragment pixels farther than r (in x or y) from every race pixel."""
    ok = np.ones(len(pix), bool)
    if not race:
        return ok
    x, y = pix.astype(np.int64) >> 8, pix.astype(np.int64) & 255
    for p in race:
        ok &= ~((np.abs(x - (p >> 8)) <= r) & (np.abs(y - (p & 255)) <= r))
    return ok


@pytest.mark.parametrize("case_name", ["small_case", "ref_size_case"])
def test_evaluation_matches_reference(request, tdi, synth, O, case_name):
    """One image-term evaluation: render (fill_diffuse_component_and_populate_texture_and_shape,
    fill_tex_im1, the convolution, fill_grads), neighbour maps (the sorts, fill_ksides,
    fill_krels, fill_krels2), Jacobian rows (render_expression_basis_texture_colmajor_rotated2_
    via_object, phase1, dI_depsilon_userotated) and the cuBLAS normal equations, on the oracle's
    geometry and rotation. Bit-equal to the oracle (and so to the product) away from painter
    races; H, g and the correlation within FP32 accumulation error."""
    case = request.getfixturevalue(case_name)
    m, fr, om = case
    K, KT = m.n_expr, m.n_expr + 6
    fs = O.FrameSet(fr)
    ocfg = O.config()
    lam = np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1))
    L = float(synth.L_INTENSITY)
    model = tdi.Model(m)
    batch = tdi.Batch(model, fr.n_frames)
    batch.set_frames(fr)
    batch.set_state(fr.state_init, lam, np.full(fr.n_frames, L, np.float32))
    batch.evaluate(tdi.default_config())
    rs = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75], nofma=True)
    for i in range(fr.n_frames):
        x = fr.state_init[i]
        geo, _ = O.vertex_stage(om, x, fr.cam[i])
        R, dR = O.rotation(x[K + 3:])
        ref = rs.evaluate(geo, R, dR, x[K:K + 3], lam[i], L, fr.cam[i], fr.target[i], *fr.x0y0[i], tau_img=25.0)
        o = O.evaluate(om, fs, i, ocfg, x, lam[i], L)
        it = O.image_terms(om, fs, i, ocfg, x, lam[i], L)
        N = o["N"]
        assert ref["N"] == N
        assert np.array_equal(ref["pix"], o["pix"]) and np.array_equal(ref["tri"], o["tri"])
        assert np.array_equal(_bits(ref["shade"]), _bits(o["sh"][0]))
        assert np.array_equal(ref["nb"], o["nb"])
        race = _race_pixels(o)
        far = _far_from(o["pix"], race, 8)
        print(f"frame {i}: N={N}, race pixels {len(race)}, fragments compared bit for bit {far.sum()}")
        assert far.sum() >= 0.9 * N
        for q in range(7):
            assert np.array_equal(_bits(ref["grads"][q][far]), _bits(o["grads"][q][far])), q
        assert np.array_equal(_bits(ref["J"][far]), _bits(o["J"][far]))
        # the product's gradients and rows equal the reference's on the same fragments
        gr = batch.read(i, tdi.READ_GRADIENTS)
        for gi, q in ((0, 0), (1, 1), (2, 2), (3, 5), (4, 6)):
            assert np.array_equal(_bits(gr[gi][far]), _bits(ref["grads"][q][far])), gi
        assert np.array_equal(_bits(batch.read(i, tdi.READ_JACOBIAN)[far]), _bits(ref["J"][far]))
        # image away from the races (blur radius 7)
        img_ok = np.ones(65536, bool)
        xs, ys = np.arange(65536) >> 8, np.arange(65536) & 255
        for p in race:
            img_ok &= ~((np.abs(xs - (p >> 8)) <= 7) & (np.abs(ys - (p & 255)) <= 7))
        assert np.array_equal(_bits(ref["image"][img_ok]), _bits(o["image"][img_ok]))
        # cuBLAS sums against the oracle's FP64 sums
        H, Ho = ref["H"].astype(np.float64), it["H"].astype(np.float64)
        eh = np.linalg.norm(H - Ho) / np.linalg.norm(Ho)
        eg = np.abs(ref["g"] - it["g"]).max() / np.abs(it["g"]).max()
        ec = abs(ref["corr"] - 25.0 * it["corr"]) / abs(25.0 * it["corr"])
        print(f"frame {i}: cuBLAS vs FP64 sums: H {eh:.2e}, g {eg:.2e}, correlation {ec:.2e}")
        if not race:
            assert eh <= 1e-4 and eg <= 1e-4 and ec <= 1e-5


def test_evaluation_against_reference_built_with_contraction(synth, O, small_case):
    """The same evaluation with the reference compiled as its CMake build compiles it (FMA
    contraction): the Jacobian rows and normal equations stay within FP32 rounding noise of
    the uncontracted oracle (relative 1e-3 on H, which a single flipped edge fragment can
    move)."""
    m, fr, om = small_case
    K = m.n_expr
    fs = O.FrameSet(fr)
    lam = np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1))
    L = float(synth.L_INTENSITY)
    rs = refpin.RefSession(m, synth.KERNEL_SIGMA_TAPS[0.75], nofma=False)
    for i in range(fr.n_frames):
        x = fr.state_init[i]
        geo, _ = O.vertex_stage(om, x, fr.cam[i])
        R, dR = O.rotation(x[K + 3:])
        ref = rs.evaluate(geo, R, dR, x[K:K + 3], lam[i], L, fr.cam[i], fr.target[i], *fr.x0y0[i], tau_img=25.0)
        it = O.image_terms(om, fs, i, O.config(), x, lam[i], L)
        eh = np.linalg.norm(ref["H"].astype(np.float64) - it["H"]) / np.linalg.norm(it["H"].astype(np.float64))
        eg = np.abs(ref["g"] - it["g"]).max() / np.abs(it["g"]).max()
        print(f"frame {i}: contracted build vs oracle: N {ref['N']} vs {it['N']}, H {eh:.2e}, g {eg:.2e}")
        assert abs(ref["N"] - it["N"]) <= 0.005 * it["N"]
        assert eh <= 1e-3 and eg <= 1e-2
