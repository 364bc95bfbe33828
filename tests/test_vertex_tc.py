"""The tensor-core vertex stage (tdi_fit_config.vertex_stage = 1): basis x coefficients as
split-BF16 products on tcgen05 with FP32 accumulation, in place of the exact stage's sequential
FP32 fused multiply-add chains (renderer.cu:806-861 forms the product with cublasSgemv).

Vertex positions against an FP64 evaluation of mean + E eps, with the bound of FP32 summation
of the K products stated in the test; projections against the exact stage; fits in the mixed
mode against the exact fits at objective and pose level."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U = 2.0 ** -24


def _pose_difference(x, x_ref, K):
    """max(|tau - tau_ref|_inf / |tau_z ref|, |u - u_ref|_inf in radians)."""
    dt = np.abs(x[K:K + 3] - x_ref[K:K + 3]).max() / abs(float(x_ref[K + 2]))
    du = np.abs(x[K + 3:K + 6] - x_ref[K + 3:K + 6]).max()
    return float(max(dt, du))


def _setup(tdi, case, synth):
    tdi.require_gpu()
    m, fr, om = case
    model = tdi.Model(m)
    batch = tdi.Batch(model, fr.n_frames)
    batch.set_frames(fr)
    lam = np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1))
    L = np.full(fr.n_frames, synth.L_INTENSITY, np.float32)
    return model, batch, lam, L


@pytest.mark.parametrize("case_name", ["small_case", "full_case"])
def test_tensor_vertex_stage_within_fp32_summation_error(request, tdi, synth, case_name):
    """|X0 - X0_fp64| <= 2 (K + 1) u (|mean| + sum_k |E_k eps_k|) per vertex and coordinate
    (u = 2^-24: the classical bound of FP32 summation of K + 1 terms, doubled for the BF16
    split's dropped pieces); the exact stage meets the same bound. Projections stay within
    1e-3 px of the exact stage's."""
    case = request.getfixturevalue(case_name)
    m, fr, om = case
    model, batch, lam, L = _setup(tdi, case, synth)
    K = m.n_expr
    batch.set_state(fr.state_init, lam, L)
    geo = {}
    for mode in (tdi.VERTEX_EXACT, tdi.VERTEX_TENSOR):
        batch.evaluate(tdi.default_config(vertex_stage=mode))
        geo[mode] = [batch.read(i, tdi.READ_GEOMETRY).reshape(6, -1) for i in range(fr.n_frames)]
    E = m.E.astype(np.float64)                      # [V, 3, K]
    worst = {tdi.VERTEX_EXACT: 0.0, tdi.VERTEX_TENSOR: 0.0}
    for i in range(fr.n_frames):
        eps = fr.state_init[i, :K].astype(np.float64)
        X64 = m.mean.astype(np.float64) + np.einsum("vck,k->cv", E, eps)
        S = np.abs(m.mean.astype(np.float64)) + np.einsum("vck,k->cv", np.abs(E), np.abs(eps))
        bound = 2 * (K + 1) * U * S
        for mode in worst:
            err = np.abs(geo[mode][i][:3].astype(np.float64) - X64)
            worst[mode] = max(worst[mode], float((err / bound).max()))
        dp = np.abs(geo[tdi.VERTEX_TENSOR][i][3:5] - geo[tdi.VERTEX_EXACT][i][3:5]).max()
        assert dp <= 1e-3, dp
        assert not np.array_equal(geo[tdi.VERTEX_TENSOR][i][:3], geo[tdi.VERTEX_EXACT][i][:3]) or K == 0
    print("vertex error / FP32 summation bound: exact", worst[tdi.VERTEX_EXACT], "tensor", worst[tdi.VERTEX_TENSOR])
    assert worst[tdi.VERTEX_EXACT] <= 1.0 and worst[tdi.VERTEX_TENSOR] <= 1.0


def test_tensor_vertex_fit_reaches_the_exact_fits_objective(tdi, synth, small_case):
    """Fits with the tensor-core vertex stage (and with both contractions on the tensor cores)
    rasterise rounding-level different vertex positions, so their iterates are not the exact
    fit's; they end at an objective within 0.5% of it, with the same status flags (apart from
    TDI_FLAG_FAIL: at most NITERS_SUCCESS outer iterations, a count the two can land on either
    side of), and with the pose close to the exact fit's: the larger of the translation difference
    relative to the depth and the rotation-vector difference in radians at most 1e-2 (median over
    frames; 5e-2 at most)."""
    m, fr, om = small_case
    model, batch, lam, L = _setup(tdi, small_case, synth)
    K = m.n_expr
    x0, lam0, rep0 = batch.fit_frames(fr, fr.state_init, lam, L, tdi.default_config(max_iters_rigid=10))
    for kw in (dict(vertex_stage=tdi.VERTEX_TENSOR),
               dict(vertex_stage=tdi.VERTEX_TENSOR, normal_eq=tdi.NORMAL_EQ_TENSOR)):
        x1, lam1, rep1 = batch.fit_frames(fr, fr.state_init, lam, L, tdi.default_config(max_iters_rigid=10, **kw))
        pose_err = []
        for i in range(fr.n_frames):
            assert (rep1[i].flags | tdi.FLAG_FAIL) == (rep0[i].flags | tdi.FLAG_FAIL)
            assert abs(rep1[i].objective - rep0[i].objective) <= 5e-3 * abs(rep0[i].objective)
            pose_err.append(_pose_difference(x1[i], x0[i], K))
        print(kw, "pose relative difference per frame:", pose_err)
        assert np.median(pose_err) <= 1e-2 and max(pose_err) <= 5e-2


def test_tensor_vertex_stage_rejects_wide_models(tdi, synth):
    """More than 80 expression components: the tensor-core vertex stage is refused with a
    message (the exact stage takes them)."""
    tdi.require_gpu()
    m = synth.make_model(500, 900, 0, n_expr=81)
    model = tdi.Model(m)
    fr = synth.make_frames(m, 1, 0, image_wh=(256, 256), tz=0.6)
    fr.target = np.zeros((1, tdi.NPIX), np.float32)
    batch = tdi.Batch(model, 1)
    batch.set_frames(fr)
    batch.set_state(fr.state_init, np.tile(synth.LAMBDA_INIT, (1, 1)), np.full(1, synth.L_INTENSITY, np.float32))
    with pytest.raises(tdi.TdiError, match="80 expression components"):
        batch.evaluate(tdi.default_config(vertex_stage=tdi.VERTEX_TENSOR))
