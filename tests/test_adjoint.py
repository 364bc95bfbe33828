"""The differentiable render loss (3di_b200.autograd, tdi_batch_loss / tdi_batch_loss_backward):
the hand-written adjoint against central finite differences of an independent FP64 forward
(numpy, the same frozen fragments) on random directions, the loss value against it, the
torch.autograd path, and the reference's own gradient (its warp-only Jacobian contracted with
the residual, derivative_computer.cu:157-164, through the pinned oracle)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _blur(img, taps):
    from scipy.ndimage import correlate1d
    k = np.asarray(taps, np.float32).astype(np.float64)[::-1]                 # the sum weights tap[7 - j] at offset j
    a = correlate1d(img.reshape(256, 256), k, axis=1, mode="constant")
    return correlate1d(a, k, axis=0, mode="constant").reshape(-1)


def _loss_np(m, fd, target, frags, z, taps):
    """FP64 loss of a frame at z = (x [K+6], lam [3], L) over the frozen fragments; fd is the
    frame's data as the batch holds it (camera, crop origin), target its 256x256 crop."""
    from scipy.spatial.transform import Rotation
    K = m.n_expr
    x, lam, L = z[:K + 6], z[K + 6:K + 9], z[K + 9]
    P0 = m.mean.astype(np.float64) + np.einsum("vck,k->cv", m.E.astype(np.float64), x[:K])
    Rm = Rotation.from_rotvec(x[K + 3:K + 6]).as_matrix()
    X = Rm @ P0 + x[K:K + 3, None]
    ph, pv, cx, cy = fd["cam"].astype(np.float64)
    xp, yp = ph * X[0] / X[2] + cx, pv * X[1] / X[2] + cy
    pix = frags["pix"].astype(np.int64)
    tri = frags["tri"]
    ib, ic, ia = m.tl[0, tri], m.tl[1, tri], m.tl[2, tri]
    sx = fd["x0"] + (pix >> 8)
    sy = fd["y0"] + (pix & 255)
    v0x, v0y = xp[ib] - xp[ia], yp[ib] - yp[ia]
    v1x, v1y = xp[ic] - xp[ia], yp[ic] - yp[ia]
    v2x, v2y = sx - xp[ia], sy - yp[ia]
    D = v0x * v1y - v0y * v1x
    al = (v2x * v1y - v2y * v1x) / D
    be = (v0x * v2y - v0y * v2x) / D
    ga = 1 - al - be
    nr = np.cross((P0[:, ib] - P0[:, ia]).T, (P0[:, ic] - P0[:, ia]).T)
    nh = nr / np.linalg.norm(nr, axis=1, keepdims=True)
    q = Rm.T @ (lam - x[K:K + 3])
    p = (P0[:, ib] * al + P0[:, ic] * be + P0[:, ia] * ga).T
    Id = nh @ q - np.sum(nh * p, axis=1)
    tex = m.tex.astype(np.float64)
    t = tex[ib] * al + tex[ic] * be + tex[ia] * ga
    I = t + L * t * Id
    img = np.zeros(65536)
    own = frags["owner"].astype(bool)
    img[pix[own]] = I[own]
    B = _blur(img, taps)
    T = _blur(target.astype(np.float32).astype(np.float64), taps)

    def grads(A):
        xx, yy = pix >> 8, pix & 255
        kr = np.where(xx < 255, pix + 256, 0); kl = np.where(xx > 0, pix - 256, 0)
        kb = np.where(yy < 255, pix + 1, 0); ka = np.where(yy > 0, pix - 1, 0)
        gx, gy = 0.5 * (A[kr] - A[kl]), 0.5 * (A[kb] - A[ka])
        h = 1e-16 + np.sqrt(4 * gx * gx + 4 * gy * gy)
        return 2 * gx / h, 2 * gy / h
    gxn, gyn = grads(B)
    sxn, syn = grads(T)
    return -np.sum(gxn * sxn + gyn * syn)


def _setup(tdi, synth, case):
    import torch
    tdi.require_gpu()
    m, fr, om = case
    model = tdi.Model(m)
    batch = tdi.Batch(model, fr.n_frames)
    batch.set_frames(fr)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(np.ascontiguousarray(fr.state_init, np.float32)).to(dev)
    lam = torch.from_numpy(np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1)).astype(np.float32)).to(dev)
    L = torch.full((fr.n_frames,), float(synth.L_INTENSITY), dtype=torch.float32, device=dev)
    return model, batch, x, lam, L


def test_adjoint_matches_fp64_finite_differences(tdi, synth, small_case):
    import torch
    ag = __import__("importlib").import_module("3di_b200.autograd")
    m, fr, om = small_case
    model, batch, x, lam, L = _setup(tdi, synth, small_case)
    cfg = tdi.default_config()
    taps = synth.KERNEL_SIGMA_TAPS[0.75]
    loss = ag.render_loss(batch, x, lam, L, cfg)
    gx, glam, gL = ag.loss_gradients(batch, cfg, x, lam, L, torch.ones_like(loss))
    K = m.n_expr
    rng = np.random.default_rng(17)
    worst = 0.0
    for i in range(fr.n_frames):
        frags = batch.read(i, tdi.READ_FRAGMENTS)
        fd = batch.read(i, tdi.READ_FRAME_DATA)
        z0 = np.concatenate([x[i].cpu().numpy(), lam[i].cpu().numpy(), [L[i].item()]]).astype(np.float64)
        f0 = _loss_np(m, fd, fr.target[i], frags, z0, taps)
        assert abs(f0 - loss[i].item()) <= 1e-10 * abs(f0), (f0, loss[i].item())
        g = np.concatenate([gx[i].cpu().numpy(), glam[i].cpu().numpy(), [gL[i].item()]])
        def central(d, h):
            return (_loss_np(m, fd, fr.target[i], frags, z0 + h * d, taps)
                    - _loss_np(m, fd, fr.target[i], frags, z0 - h * d, taps)) / (2 * h)

        for _ in range(32 // fr.n_frames + 1):
            d = rng.normal(size=g.shape)
            d /= np.linalg.norm(d)
            # Richardson extrapolation of two central differences cancels the h^2 term
            h = 1e-5
            d1, d2 = central(d, h), central(d, h / 2)
            fdv = (4.0 * d2 - d1) / 3.0
            rel = abs(float(g @ d) - fdv) / max(abs(fdv), 1e-3 * np.linalg.norm(g))
            if rel > worst:
                worst, info = rel, (i, float(g @ d), fdv, d1, d2)
    print("adjoint vs FP64 central differences (Richardson): worst relative error", worst, info)
    assert worst <= 1e-6


def test_autograd_function_gives_the_adjoint(tdi, synth, small_case):
    import torch
    ag = __import__("importlib").import_module("3di_b200.autograd")
    model, batch, x, lam, L = _setup(tdi, synth, small_case)
    xr, lr, Lr = (t.clone().requires_grad_(True) for t in (x, lam, L))
    loss = ag.render_loss(batch, xr, lr, Lr)
    (2.0 * loss).sum().backward()
    gx, glam, gL = ag.loss_gradients(batch, tdi.default_config(), x, lam, L, torch.full_like(loss, 2.0))
    assert xr.grad.dtype == torch.float32
    torch.testing.assert_close(xr.grad.double(), gx.float().double(), rtol=1e-6, atol=0)
    torch.testing.assert_close(lr.grad.double(), glam.float().double(), rtol=1e-6, atol=0)


def test_adjoint_against_the_references_gradient(tdi, synth, O, small_case):
    """The reference's gradient of its image term is its warp-only Jacobian contracted with the
    residual (no blur, shading or barycentric derivatives, approximate neighbours); here through
    the oracle pinned to the reference's kernels. It points the same way as the exact gradient
    over the pose and overall: cosine at least 0.9 (0.96-0.99 measured on these frames)."""
    import torch
    ag = __import__("importlib").import_module("3di_b200.autograd")
    m, fr, om = small_case
    model, batch, x, lam, L = _setup(tdi, synth, small_case)
    cfg = tdi.default_config()
    gx, _, _ = ag.loss_gradients(batch, cfg, x, lam, L, torch.ones(fr.n_frames, dtype=torch.float64, device=x.device))
    fs = O.FrameSet(fr)
    K = m.n_expr
    for i in range(fr.n_frames):
        it = O.image_terms(om, fs, i, O.config(), x[i].cpu().numpy(), lam[i].cpu().numpy(), float(L[i].item()))
        gref = it["g"].astype(np.float64)                 # = -25 sum(gxs Gx + gys Gy) = 25 dL/dtheta (warp-only)
        gad = 25.0 * gx[i].cpu().numpy()
        cos_all = gref @ gad / (np.linalg.norm(gref) * np.linalg.norm(gad))
        cos_pose = gref[K:] @ gad[K:] / (np.linalg.norm(gref[K:]) * np.linalg.norm(gad[K:]))
        print(f"frame {i}: cosine(reference J^T r, adjoint) all {cos_all:.4f}, pose {cos_pose:.4f}")
        assert cos_pose >= 0.9 and cos_all >= 0.9
