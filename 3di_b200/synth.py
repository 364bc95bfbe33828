"""Seeded synthetic morphable model and video frames for the 3DMM fitting path.

The BFM'09 files that 3DI fits with are licence-gated and absent, so every input here
is generated from a seed with the shapes and value distributions of the real model:

* units: the reference's model units, in which the inter-ocular distance is 89 units
  (~63 mm, build/models/prepare_BFM.py:260-261), so that every unit-bearing constant of the
  reference (the orthographic start sigma = 15, the initial light position and intensity, the
  landmark initializer's slack) meets the scale it was tuned for; sizes below are quoted in
  metres and converted with ``UNIT_M``;
* geometry: ``V`` vertices on a face-like ellipsoid cap (half-axes a=0.08 m, b=0.10 m,
  depth c=0.05 m; the cap bulges toward the camera) with a nose, eye sockets and a brow
  ridge, Delaunay-triangulated and trimmed to ``T`` triangles by dropping the outermost ones;
* bases: smooth Gaussian random fields (a handful of random cosine modes each, spatial
  frequency rising slowly with the component index k), scaled so every component has
  standard deviation ``0.006 / k`` m (k = 1-based); the deformed meshes stay unfolded like
  a real face mesh (total projected triangle area within ~10% of the covered area);
  79 expression components and 199 identity components; the albedo is 0.62 plus a
  mottled random field, darker at the eyes, brows, nostrils and lips;
* the subject is mean + identity deformation, fixed for the video fit, exactly like the
  ``.shp``/``.tex`` identity files that ``video_from_saved_identity`` loads
  (src/apps/video_from_saved_identity.cu:141-150);
* frames: pinhole camera f=800 px at the original resolution, yaw/pitch/roll in degrees,
  51 landmark vertices chosen by farthest-point sampling and projected with Gaussian
  pixel noise.

The reference rescales every frame so the landmark box is ``REF_FACE_SIZE`` px
(src/lib/video_fitter.cu:355-360, src/lib/camera.h:162-174) and fits a 256x256 crop whose
origin is ``max(min_landmark - size/1.5, 0)`` (src/lib/renderer.cu:585-607). The
generator performs that rescaling on the camera and emits frames directly in the
rescaled coordinate system; the target crop itself is rendered by a caller-supplied
renderer (``render_fn``), so this module needs no GPU and no CPU renderer.

Streams: numpy PCG64 with seed ``1000*config_id + stream`` (0 geometry/bases,
1 coefficients/pose, 2 noise, 3 face boxes).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

NL = 51                # landmarks per frame (src/lib/constants.h:31)
DIM = 256              # crop side (src/lib/constants.h:55-56)
REF_FACE_SIZE = 78.0   # build/configs/BFMmm-19830.cfg1.global4.txt:8
KERNEL_SIGMA_TAPS = {  # 15-tap tables, src/lib/video_fitter.cu:53-56
    0.50: [2.15799964e-43, 4.23189662e-32, 1.51709817e-22, 9.96126162e-15, 1.19794565e-08,
           2.63865077e-04, 1.06450766e-01, 7.86570668e-01, 1.06450766e-01, 2.63865077e-04,
           1.19794565e-08, 9.96126162e-15, 1.51709817e-22, 4.23189662e-32, 2.15799964e-43],
    2.00: [4.9640312e-06, 8.9220186e-05, 1.0281866e-03, 7.5973268e-03, 3.5993993e-02,
           1.0934010e-01, 2.1296541e-01, 2.6596162e-01, 2.1296541e-01, 1.0934010e-01,
           3.5993993e-02, 7.5973268e-03, 1.0281866e-03, 8.9220186e-05, 4.9640312e-06],
    0.75: [6.4550189e-20, 6.7361578e-15, 1.1880850e-10, 3.5416286e-07, 1.7843490e-04,
           1.5194189e-02, 2.1867350e-01, 5.3190696e-01, 2.1867350e-01, 1.5194189e-02,
           1.7843490e-04, 3.5416286e-07, 1.1880850e-10, 6.7361578e-15, 6.4550189e-20],
    1.00: [9.1347208e-12, 6.0758834e-09, 1.4867194e-06, 1.3383022e-04, 4.4318484e-03,
           5.3990968e-02, 2.4197073e-01, 3.9894229e-01, 2.4197073e-01, 5.3990968e-02,
           4.4318484e-03, 1.3383022e-04, 1.4867194e-06, 6.0758834e-09, 9.1347208e-12],
}
# One model unit in metres: the inter-ocular distance is 89 units (~63 mm,
# build/models/prepare_BFM.py:260-261). Initial light position and intensity of a video fit
# (src/lib/video_fitter.cu:115-116) in those units; the intensity is held fixed by the video fit.
UNIT_M = 0.063 / 89.0
LAMBDA_INIT = np.array([-7.3627, 51.1364, 100.1784], dtype=np.float32)
L_INTENSITY = np.float32(0.005)


def _rng(config_id: int, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(1000 * config_id + stream))


@dataclasses.dataclass
class Model:
    """A morphable model in the layouts the fitting library takes.

    mean   [3, V]   subject shape (identity applied), planes X, Y, Z
    E      [V, 3, K] expression basis, row-major per vertex and coordinate
    tex    [V]      subject albedo
    tl     [3, T]   0-based triangle vertex ids, planes (as ``tl.dat`` columns minus 1)
    lis    [51]     landmark vertex ids
    eps_lb/eps_ub   expression bounds of the shape fit; *_ft those of the finetune
    """
    mean: np.ndarray
    E: np.ndarray
    tex: np.ndarray
    tl: np.ndarray
    lis: np.ndarray
    eps_lb: np.ndarray
    eps_ub: np.ndarray
    eps_lb_ft: np.ndarray
    eps_ub_ft: np.ndarray

    @property
    def n_vertices(self) -> int:
        return self.mean.shape[1]

    @property
    def n_triangles(self) -> int:
        return self.tl.shape[1]

    @property
    def n_expr(self) -> int:
        return self.E.shape[2]


@dataclasses.dataclass
class Frames:
    """Per-frame inputs of a fit, all float32 except the crop origin.

    xl, yl [F, 51] landmarks in the rescaled frame; bounds [F, 4, 51] (lx, ly, ux, uy)
    as fractions of the face size; face_size [F]; cam [F, 4] (phix, phiy, cx, cy);
    x0y0 [F, 2] uint16 crop origins; state_true / state_init [F, K+6] (epsilon, tau, u);
    lam_true [F, 3]; target [F, 256*256] column-major crops (filled by ``render_targets``).
    """
    xl: np.ndarray
    yl: np.ndarray
    bounds: np.ndarray
    face_size: np.ndarray
    cam: np.ndarray
    x0y0: np.ndarray
    state_true: np.ndarray
    state_init: np.ndarray
    lam_true: np.ndarray
    target: np.ndarray | None = None

    @property
    def n_frames(self) -> int:
        return self.xl.shape[0]


def _blob(u, v, cu, cv, su, sv):
    """Gaussian bump of height 1 centred at (cu, cv) with half-widths (su, sv) in (u, v)."""
    return np.exp(-(((u - cu) / su) ** 2 + ((v - cv) / sv) ** 2))


def _face_relief(u, v):
    """Height of nose ridge and tip, eye sockets and brow ridge toward the camera (metres)."""
    r = 0.022 * _blob(u, v, 0.0, -0.08, 0.085, 0.24) + 0.006 * _blob(u, v, 0.0, -0.28, 0.12, 0.06)
    r = r - 0.008 * (_blob(u, v, -0.33, 0.22, 0.12, 0.07) + _blob(u, v, 0.33, 0.22, 0.12, 0.07))
    r = r + 0.004 * (_blob(u, v, -0.33, 0.40, 0.16, 0.05) + _blob(u, v, 0.33, 0.40, 0.16, 0.05))
    return r


def _smooth_fields(rng, uv, n_fields, std, n_modes=5, s_hi=0.04):
    """n_fields smooth random fields over points uv [V,2], each with per-point std ``std[i]``;
    the spatial frequency of field k (1-based) has scale 0.25 + s_hi * sqrt(k) cycles per
    unit of (u, v)."""
    V = uv.shape[0]
    out = np.empty((n_fields, V), dtype=np.float64)
    for i in range(n_fields):
        k = i + 1
        s = 0.25 + s_hi * math.sqrt(k)
        f = rng.normal(0.0, s, size=(n_modes, 2))
        ph = rng.uniform(0, 2 * math.pi, size=n_modes)
        w = rng.normal(0.0, 1.0, size=n_modes)
        field = np.cos(2 * math.pi * (uv @ f.T) + ph) @ w
        field -= field.mean()
        sd = field.std()
        out[i] = field * (std[i] / (sd if sd > 0 else 1.0))
    return out


def _face_albedo(rng, uv, u, v, beta, n_tex):
    """Skin albedo with a mottled random field, darker at the eyes, brows, nostrils and lips."""
    tex = 0.62 + beta @ _smooth_fields(rng, uv, n_tex, 0.05 / np.sqrt(np.arange(1, n_tex + 1)), s_hi=0.25)
    tex = tex - 0.40 * (_blob(u, v, -0.33, 0.22, 0.09, 0.04) + _blob(u, v, 0.33, 0.22, 0.09, 0.04))
    tex = tex - 0.30 * (_blob(u, v, -0.33, 0.40, 0.14, 0.025) + _blob(u, v, 0.33, 0.40, 0.14, 0.025))
    tex = tex - 0.25 * (_blob(u, v, -0.07, -0.25, 0.03, 0.02) + _blob(u, v, 0.07, -0.25, 0.03, 0.02))
    tex = tex - 0.30 * _blob(u, v, 0.0, -0.48, 0.20, 0.035)
    tex = np.clip(tex, 0.05, 1.0)
    return tex


def _basis_std(K, rough=False):
    k = np.arange(1, K + 1, dtype=np.float64)
    return 0.01 * k ** -0.5 if rough else 0.006 / k


def make_model(n_vertices: int, n_triangles: int, config_id: int = 0, n_expr: int = 79,
               n_id: int = 199, n_tex: int = 199, eps_bound: float = 4.5,
               finetune_coef: float = 2.75, surface: str = "face") -> Model:
    """Seeded face-like model with ``n_vertices`` points and ``n_triangles`` triangles.

    ``surface="face"`` (default): smooth bases with std 0.006/k m, a relief (nose, eye
    sockets, brows) and albedo features; deformed meshes stay unfolded. ``surface="rough"``:
    bases with std 0.01*k**-0.5 m and faster-rising spatial frequency, plain cap and albedo
    0.6 plus fields of the same std; its deformed meshes fold over themselves (total
    projected triangle area several times the covered area, about half the triangles facing
    away), which gives the raster many more overlapping fragments per pixel.
    """
    if surface not in ("face", "rough"):
        raise ValueError(surface)
    rough = surface == "rough"
    from scipy.spatial import Delaunay

    rng = _rng(config_id, 0)
    a, b, c = 0.08, 0.10, 0.05
    rmax = 0.97
    V = n_vertices
    i = np.arange(V, dtype=np.float64) + 0.5
    r = rmax * np.sqrt(i / V)
    th = i * math.pi * (3.0 - math.sqrt(5.0))
    spacing = math.sqrt(math.pi / V) * rmax
    r = np.clip(r + rng.uniform(-0.12, 0.12, V) * spacing * 0.5, 0.0, rmax)
    th = th + rng.uniform(-0.12, 0.12, V) * spacing / np.maximum(r, spacing)
    u = r * np.cos(th)
    v = r * np.sin(th)
    x = a * u
    y = b * v
    # cap bulging toward the camera (-z), with a face's relief: nose ridge and tip, eye
    # sockets, brow ridge (metres)
    z = -c * np.sqrt(np.maximum(1.0 - u * u - v * v, 0.0))
    if not rough:
        z = z - _face_relief(u, v)

    tri = Delaunay(np.c_[u, v]).simplices.astype(np.int64)
    if tri.shape[0] < n_triangles:
        raise ValueError(f"Delaunay gave {tri.shape[0]} triangles, fewer than {n_triangles}")
    cen = np.sqrt(u[tri].mean(1) ** 2 + v[tri].mean(1) ** 2)
    keep = np.sort(np.argsort(cen, kind="stable")[:n_triangles])
    tri = tri[keep]
    # Delaunay simplices are counter-clockwise in (u, v); the reference's face normal is
    # (v0 - v2) x (v1 - v2) (src/lib/newfuncs.cu:99-117). Swap two columns so that normal
    # points toward the camera (-z in object space).
    tri = tri[:, [0, 2, 1]]
    # Shuffle triangle order with a fixed permutation so neighbouring triangles do not sit in
    # neighbouring slots (the real tl.dat order is not spatially sorted either).
    tri = tri[rng.permutation(tri.shape[0])]

    uv = np.c_[u, v]
    E = np.empty((V, 3, n_expr), dtype=np.float64)
    s_hi = 0.22 if rough else 0.04
    std_e = _basis_std(n_expr, rough)
    for cidx in range(3):
        E[:, cidx, :] = _smooth_fields(rng, uv, n_expr, std_e, s_hi=s_hi).T
    # Identity: only the subject's deformation is needed (identity is fixed in the fit).
    std_i = _basis_std(n_id, rough)
    alpha = np.clip(rng.normal(size=n_id), -3.5, 3.5)
    ident = np.zeros((3, V))
    for cidx in range(3):
        ident[cidx] = alpha @ _smooth_fields(rng, uv, n_id, std_i, s_hi=s_hi)
    beta = np.clip(rng.normal(size=n_tex), -3.5, 3.5)
    if rough:
        tex = 0.6 + beta @ _smooth_fields(rng, uv, n_tex, _basis_std(n_tex, True), s_hi=s_hi)
    else:
        tex = _face_albedo(rng, uv, u, v, beta, n_tex)

    mean = (np.stack([x, y, z]) + ident) / UNIT_M
    E = E / UNIT_M

    # 51 landmarks by farthest-point sampling over the cap, starting at the centre.
    pts = np.c_[u, v]
    lis = [int(np.argmin(u * u + v * v))]
    d = np.sum((pts - pts[lis[0]]) ** 2, axis=1)
    for _ in range(NL - 1):
        j = int(np.argmax(d))
        lis.append(j)
        d = np.minimum(d, np.sum((pts - pts[j]) ** 2, axis=1))

    lb = np.full(n_expr, -eps_bound, dtype=np.float32)
    ub = np.full(n_expr, eps_bound, dtype=np.float32)
    return Model(mean=mean.astype(np.float32), E=E.astype(np.float32),
                 tex=tex.astype(np.float32), tl=np.ascontiguousarray(tri.T.astype(np.int32)),
                 lis=np.array(lis, dtype=np.int32), eps_lb=lb, eps_ub=ub,
                 eps_lb_ft=(lb * np.float32(finetune_coef)).astype(np.float32),
                 eps_ub_ft=(ub * np.float32(finetune_coef)).astype(np.float32))


def euler_to_axis_angle(yaw, pitch, roll):
    """Axis-angle u of R = Rz(roll) Ry(yaw) Rx(pitch) (angles in radians)."""
    cx, sx = math.cos(pitch), math.sin(pitch)
    cy, sy = math.cos(yaw), math.sin(yaw)
    cz, sz = math.cos(roll), math.sin(roll)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    R = Rz @ Ry @ Rx
    th = math.acos(max(-1.0, min(1.0, (np.trace(R) - 1) / 2)))
    w = np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]])
    return w * (th / (2 * math.sin(th))) if th > 1e-9 else np.array([1e-6, 0.0, 0.0])


def rodrigues(u):
    th = float(np.linalg.norm(u))
    n = np.asarray(u, dtype=np.float64) / th
    S = np.array([[0, -n[2], n[1]], [n[2], 0, -n[0]], [-n[1], n[0], 0]])
    return np.eye(3) + math.sin(th) * S + (1 - math.cos(th)) * (S @ S)


def crop_origin(xl, yl):
    """Crop origin from rescaled landmarks, as Renderer::set_x0_short_y0_short with padding
    (src/lib/renderer.cu:580-598): (ushort) max<float>(min - size/1.5, 0) with the
    subtraction done in double."""
    xl = np.asarray(xl, np.float32)
    yl = np.asarray(yl, np.float32)
    sz = np.float32(max(np.float32(xl.max() - xl.min()), np.float32(yl.max() - yl.min())))
    x0 = np.float32(float(xl.min()) - float(sz) / 1.5)
    y0 = np.float32(float(yl.min()) - float(sz) / 1.5)
    return int(max(x0, np.float32(0))), int(max(y0, np.float32(0)))


def face_size(xl, yl):
    """max(width, height) of the landmark box (src/lib/funcs.cu:44-54), float32."""
    xl = np.asarray(xl, np.float32)
    yl = np.asarray(yl, np.float32)
    return np.float32(max(np.float32(xl.max() - xl.min()), np.float32(yl.max() - yl.min())))


def make_frames(model: Model, n_frames: int, config_id: int = 0, image_wh=(256, 256),
                tz: float = 0.6, box_range=None, ar1: bool = False,
                angle_range_deg: float = 30.0, focal: float = 800.0,
                lmk_noise_px: float = 1.5, init_pose_noise: float = 1.0,
                bound: float = 0.08, margin: float = 0.03) -> Frames:
    """Per-frame cameras, poses, landmarks and initial states.

    ``box_range`` (px at the original resolution) draws the landmark-box size per frame and
    sets tz from it; otherwise tz is fixed (``tz`` in metres). ``ar1`` gives an AR(1) expression sequence
    (rho 0.95, unit marginal variance) and random-walk angles clamped to +-40 deg, else
    independent draws. Initial states stand in for the landmark initializer: ground truth
    state perturbed by ``init_pose_noise`` times (2 deg, 3 mm, 0.3 per expression),
    shrunk until the landmark constraints hold strictly.
    """
    rng = _rng(config_id, 1)
    rng_noise = _rng(config_id, 2)
    rng_box = _rng(config_id, 3)
    K = model.n_expr
    W, H = image_wh
    F = n_frames
    lis = model.lis
    mean = model.mean.astype(np.float64)
    Eland = model.E[lis].astype(np.float64)          # [51, 3, K]

    eps = np.empty((F, K))
    ang = np.empty((F, 3))
    if ar1:
        rho = 0.95
        e = rng.normal(size=K)
        a = rng.uniform(-20, 20, size=3)
        for f in range(F):
            if f:
                e = rho * e + math.sqrt(1 - rho * rho) * rng.normal(size=K)
                a = np.clip(a + rng.normal(0.0, 1.5, size=3), -40.0, 40.0)
            eps[f] = e
            ang[f] = a
    else:
        eps[:] = rng.normal(size=(F, K))
        ang[:] = rng.uniform(-angle_range_deg, angle_range_deg, size=(F, 3))
    eps = np.clip(eps, -3.5, 3.5)

    xl_all = np.empty((F, NL), np.float32)
    yl_all = np.empty((F, NL), np.float32)
    cams = np.empty((F, 4), np.float32)
    fs_all = np.empty(F, np.float32)
    x0y0 = np.empty((F, 2), np.uint16)
    st_true = np.zeros((F, K + 6), np.float32)
    st_init = np.zeros((F, K + 6), np.float32)
    lam_true = np.empty((F, 3), np.float32)
    extent = float(max(np.ptp(mean[0, lis]), np.ptp(mean[1, lis])))

    dx = 2 * bound
    bl = -bound - margin * dx
    bu = bound + margin * dx
    Eall = model.E.astype(np.float64)
    for f in range(F):
        yaw, pitch, roll = np.deg2rad(ang[f])
        u = euler_to_axis_angle(yaw, pitch, roll)
        R = rodrigues(u)
        if box_range is not None:
            box = rng_box.uniform(*box_range)
            tzf = focal * extent / box
        else:
            tzf = tz / UNIT_M
        # face centre somewhere inside the frame, away from the borders
        half = focal * extent / tzf * 0.75
        px = rng_box.uniform(min(half, W / 2), max(W - half, W / 2))
        py = rng_box.uniform(min(half, H / 2), max(H - half, H / 2))
        cx0, cy0 = W / 2.0, H / 2.0
        tx = (px - cx0) * tzf / focal
        ty = (py - cy0) * tzf / focal
        tau = np.array([tx, ty, tzf])
        P = mean[:, lis] + np.einsum("lck,k->cl", Eland, eps[f])
        Pc = R @ P + tau[:, None]
        xo = focal * Pc[0] / Pc[2] + cx0 + rng_noise.normal(0.0, lmk_noise_px, NL)
        yo = focal * Pc[1] / Pc[2] + cy0 + rng_noise.normal(0.0, lmk_noise_px, NL)
        # VideoFitter rescales by REF_FACE_SIZE over the integer landmark box
        # (src/lib/input_data.cu:123-138, src/lib/video_fitter.cu:355-360).
        box_int = max(int(xo.max()) - int(xo.min()), int(yo.max()) - int(yo.min()))
        rc = REF_FACE_SIZE / box_int
        # Pad the rescaled frame on the left/top (shift the principal point) when the face
        # would come closer than the crop margin to the frame origin, so every vertex lands
        # inside the 256x256 crop with a border to spare.
        full = R @ (mean + np.einsum("vck,k->cv", Eall, eps[f])) + tau[:, None]
        xs = (focal * full[0] / full[2] + cx0) * rc
        ys = (focal * full[1] / full[2] + cy0) * rc
        need = REF_FACE_SIZE / 1.5 + 16.0
        shx = max(0.0, need - float(xo.min() * rc), 8.0 - float(xs.min()))
        shy = max(0.0, need - float(yo.min() * rc), 8.0 - float(ys.min()))
        xl = (xo * rc + shx).astype(np.float32)
        yl = (yo * rc + shy).astype(np.float32)
        xl_all[f], yl_all[f] = xl, yl
        cams[f] = [focal * rc, focal * rc, cx0 * rc + shx, cy0 * rc + shy]
        fs_all[f] = face_size(xl, yl)
        x0y0[f] = crop_origin(xl, yl)
        if (xs.min() + shx - x0y0[f, 0] < 2 or xs.max() + shx - x0y0[f, 0] > DIM - 3
                or ys.min() + shy - x0y0[f, 1] < 2 or ys.max() + shy - x0y0[f, 1] > DIM - 3):
            raise ValueError(f"frame {f}: face does not fit the 256x256 crop")
        st_true[f, :K] = eps[f]
        st_true[f, K:K + 3] = tau
        st_true[f, K + 3:] = u
        lam_true[f] = LAMBDA_INIT + rng.normal(0.0, 0.02, 3) / UNIT_M
        # Initial state: stands in for the landmark initializer. Perturb pose and
        # expressions, halving the perturbation until every landmark constraint is
        # strictly satisfied (the barrier needs a feasible start).
        scale = init_pose_noise
        dang = rng_noise.normal(0.0, 2.0, 3)
        dtau = rng_noise.normal(0.0, 0.003, 3) / UNIT_M
        deps = rng_noise.normal(0.0, 0.3, K)
        fs = float(fs_all[f])
        for _ in range(12):
            u0 = euler_to_axis_angle(*np.deg2rad(ang[f] + dang * scale))
            t0 = tau + dtau * scale
            e0 = np.clip(eps[f] + deps * scale, -3.5, 3.5)
            R0 = rodrigues(u0)
            P0 = R0 @ (mean[:, lis] + np.einsum("lck,k->cl", Eland, e0)) + t0[:, None]
            xp0 = cams[f, 0] * P0[0] / P0[2] + cams[f, 2]
            yp0 = cams[f, 1] * P0[1] / P0[2] + cams[f, 3]
            g = np.concatenate([xp0 - (xl + bl * fs), yp0 - (yl + bl * fs),
                                (xl + bu * fs) - xp0, (yl + bu * fs) - yp0])
            if g.min() > 0.5:
                break
            scale *= 0.5
        st_init[f, :K] = e0
        st_init[f, K:K + 3] = t0
        st_init[f, K + 3:] = u0

    bnd = np.empty((F, 4, NL), np.float32)
    bnd[:, 0] = bl
    bnd[:, 1] = bl
    bnd[:, 2] = bu
    bnd[:, 3] = bu
    return Frames(xl=xl_all, yl=yl_all, bounds=bnd, face_size=fs_all, cam=cams, x0y0=x0y0,
                  state_true=st_true, state_init=st_init, lam_true=lam_true)


def add_noise(images: np.ndarray, sigma: float, config_id: int = 0) -> np.ndarray:
    rng = _rng(config_id, 2)
    return (images + rng.normal(0.0, sigma, images.shape)).astype(np.float32)


# Workloads named after what they are; sizes follow the reference's fitted model class.
WORKLOADS = {
    "cap5k_256": dict(model=dict(n_vertices=5000, n_triangles=9800, config_id=0),
                      frames=dict(config_id=0, image_wh=(256, 256), tz=0.6)),
    "cap53k_1080p": dict(model=dict(n_vertices=53490, n_triangles=106466, config_id=1),
                         frames=dict(config_id=1, image_wh=(1920, 1080), box_range=(300, 600))),
    "cap53k_video": dict(model=dict(n_vertices=53490, n_triangles=106466, config_id=1),
                         frames=dict(config_id=3, image_wh=(1920, 1080), box_range=(120, 600), ar1=True)),
}


def make_workload(name: str, n_frames: int, seed_offset: int = 0, surface: str = "face"):
    """Model and frames of a named workload; ``seed_offset`` shifts the frame seeds."""
    spec = WORKLOADS[name]
    m = make_model(**spec["model"], surface=surface)
    fkw = dict(spec["frames"])
    cid = fkw.pop("config_id") + seed_offset
    return m, make_frames(m, n_frames, cid, **fkw)
