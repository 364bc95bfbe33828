"""The subject's shape and albedo from identity and texture coefficients (tdi_apply_identity;
the reference's Renderer::compute_nonrigid_shape_identityonly and compute_texture,
renderer.cu:866-883,941-951): the oracle against FP64 within the FP32 summation bound, the
device against the oracle bit for bit, at the full model size and with empty bases."""
import numpy as np
import pytest

U = 2.0 ** -24


def _case(V, KA, KB, seed=3):
    rng = np.random.default_rng(seed)
    mean0 = (rng.normal(0, 60, (3, V))).astype(np.float32)
    I = (rng.normal(0, 1, (3, V, KA)) / np.sqrt(np.arange(1, KA + 1))).astype(np.float32)
    alpha = np.clip(rng.normal(0, 1, KA), -3.5, 3.5).astype(np.float32)
    tex0 = rng.uniform(0.3, 0.9, V).astype(np.float32)
    T = (rng.normal(0, 0.05, (V, KB)) / np.sqrt(np.arange(1, KB + 1))).astype(np.float32)
    beta = np.clip(rng.normal(0, 1, KB), -3.5, 3.5).astype(np.float32)
    return mean0, I, alpha, tex0, T, beta


def test_oracle_within_fp32_summation_bound(O):
    mean0, I, alpha, tex0, T, beta = _case(2000, 199, 199)
    mean, tex = O.apply_identity(mean0, I, alpha, tex0, T, beta)
    m64 = mean0.astype(np.float64) + np.einsum("cvk,k->cv", I.astype(np.float64), alpha.astype(np.float64))
    S = np.abs(mean0.astype(np.float64)) + np.einsum("cvk,k->cv", np.abs(I.astype(np.float64)), np.abs(alpha))
    assert np.all(np.abs(mean - m64) <= (199 + 1) * U * S)
    t64 = tex0.astype(np.float64) + T.astype(np.float64) @ beta.astype(np.float64)
    St = np.abs(tex0.astype(np.float64)) + np.abs(T.astype(np.float64)) @ np.abs(beta.astype(np.float64))
    assert np.all(np.abs(tex - t64) <= (199 + 1) * U * St)
    # empty bases: a copy
    m0, t0 = O.apply_identity(mean0, None, None, tex0, None, None)
    assert np.array_equal(m0, mean0) and np.array_equal(t0, tex0)


@pytest.mark.gpu
@pytest.mark.parametrize("V,KA,KB", [(53490, 199, 199), (5000, 199, 0), (5000, 0, 199), (37, 3, 1)])
def test_device_equals_oracle(tdi, O, V, KA, KB):
    tdi.require_gpu()
    mean0, I, alpha, tex0, T, beta = _case(V, KA, KB)
    args = (mean0, I if KA else None, alpha if KA else None, tex0, T if KB else None, beta if KB else None)
    dm, dt = tdi.apply_identity(*args)
    om, ot = O.apply_identity(*args)
    assert np.array_equal(dm.view(np.uint32), om.view(np.uint32))
    assert np.array_equal(dt.view(np.uint32), ot.view(np.uint32))
    if not KA:
        assert np.array_equal(dm, mean0)
