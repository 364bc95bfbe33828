"""Drop-in for 3DI's ``video_from_saved_identity`` executable, over this library's C ABI.

Same arguments as the reference (src/apps/video_from_saved_identity.cu:54-172)::

    python -m 3di_b200.video_from_saved_identity <video> <landmarks.txt> <config.yaml>
        <field-of-view-degrees | calibration.yaml> <identity.shp> <identity.tex>
        <out.expressions> <out.poses> <out.illums> [--models-root DIR] [--chunk N]

so that ``build/process_video.py`` can call it in place of the reference's binary. The files
it reads are the reference's:

* the YAML configuration (config.cu:350-541), read with OpenCV's FileStorage as the reference
  reads it; the keys of the fitting path are used (EXP_BASIS, MM, OPTS_DELTA_EPS,
  REF_FACE_SIZE, KERNEL_SIGMA, NRES_COEFS, TWOSTAGE_ILLUM, FINETUNE_EXPRESSIONS,
  FINETUNE_COEF, NITERS_SUCCESS, MAX_VID_FRAMES_TO_PROCESS, SKIP_FIRST_N_SECS);
* the model directory ``models/MMs/<MM>/`` (config.cu:175-192,317-331; layouts of
  build/models/prepare_BFM.py:280-307): ``E/EX_79.dat`` ... (V x K), ``tl.dat`` (T x 3,
  1-based), ``li.dat`` (51 landmark vertex ids, 0-based), ``p0L_mat.dat`` (51 x 3) and the
  expression bounds ``E/sigma_epsilons_79_{lower,upper}v2.dat`` scaled by OPTS_DELTA_EPS
  (and by FINETUNE_COEF for the finetune, logbarrier_initializer.cu:271-286);
* the subject's identity: ``.shp`` (V x 3, the shape with the identity applied) and ``.tex``
  (V x 1, the albedo), as save_identity_and_shape writes them;
* the landmarks: one row per video frame, x1 y1 x2 y2 ... x51 y51 (input_data.cu:98-121);
* the camera: a field of view in degrees (focal length cx / tan(fov / 2), principal point at
  the image centre, video_from_saved_identity.cu:96-121) or an OpenCV calibration file
  (camera.h:80-127, cameraMatrix_postUndistort).

It writes ``.expressions`` (T x 79), ``.poses`` (T x 9: tau, u, yaw, pitch, roll) and
``.illums`` (T x 4) with the reference's text layout and NaN rows for frames without a
reconstruction (3di_b200/video.py's VideoOutput).

The per-frame pipeline is VideoFitter::fit_video_frames_auto's (video_fitter.cu:116-300) for
a window of one frame: the landmark check of the original frame (a landmark fit at scale 1
that must succeed), then for each of the NRES_COEFS reference face sizes the crop, the landmark
initialisation and the image fit (tdi_batch_landmark_init, tdi_batch_fit), and the average of
the scales. Departures: frames are fitted in chunks, all scales of a chunk in one batch, so the
light position of every fit starts from the reference's initial value (video_fitter.cu:115-119)
instead of the previous frame's fit, which makes frames independent; the landmark bounds are
constant boxes of +-0.08 face sizes widened by the reference's 0.03 margin (its per-landmark
bound-estimator networks are not available); video frames are decoded with OpenCV's Python
bindings.
"""
from __future__ import annotations

import argparse
import importlib
import math
import os
import sys

import numpy as np

F32 = np.float32
NL = 51
LAMBDA0 = np.array([-7.3627, 51.1364, 100.1784], F32)    # video_fitter.cu:115-116 (model units)
L0 = F32(0.005)                                           # video_fitter.cu:560
BOX = 0.08                                                # constant landmark box (face sizes)
BOX_MARGIN = 0.03                                         # logbarrier_initializer.cu:2204-2245

DEFAULTS = dict(EXP_BASIS="GLOBAL79", OPTS_DELTA_EPS=1.1, REF_FACE_SIZE=78.0, KERNEL_SIGMA=0.5,
                NRES_COEFS=4, TWOSTAGE_ILLUM=0, FINETUNE_EXPRESSIONS=0, FINETUNE_COEF=1.5,
                NITERS_SUCCESS=6, MAX_VID_FRAMES_TO_PROCESS=50000, SKIP_FIRST_N_SECS=0.0)
BASES = {"GLOBAL79": ("E/EX_79.dat", "E/EY_79.dat", "E/EZ_79.dat",
                      "E/sigma_epsilons_79_lowerv2.dat", "E/sigma_epsilons_79_upperv2.dat"),
         "GLOBAL29": ("E/EX.dat", "E/EY.dat", "E/EZ.dat",
                      "E/sigma_epsilons_lower.dat", "E/sigma_epsilons_upper.dat")}


def read_config(path: str) -> dict:
    """The fitting path's keys of the reference's YAML configuration, with its defaults
    (config.cu:30-110) for keys the file leaves out."""
    import cv2
    fs = cv2.FileStorage(path, cv2.FILE_STORAGE_READ)
    if not fs.isOpened():
        raise FileNotFoundError(path)
    out = dict(DEFAULTS)
    for key, default in DEFAULTS.items():
        node = fs.getNode(key)
        if node.empty():
            continue
        out[key] = node.string() if isinstance(default, str) else type(default)(node.real())
    node = fs.getNode("MM")
    if node.empty():
        raise ValueError(f"{path}: no MM (model name)")
    out["MM"] = node.string()
    fs.release()
    return out


def read_matrix(path: str, ncols: int | None = None) -> np.ndarray:
    """A whitespace-separated text matrix (read2DVectorFromFile), one row per line."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if ncols is not None and a.shape[1] != ncols:
        raise ValueError(f"{path}: {a.shape[1]} columns, expected {ncols}")
    return a


def read_model(model_dir: str, cfg: dict, shp: str, tex: str):
    """The subject's morphable model in the library's layouts (3di_b200.Model's input), and the
    orthographic step's landmark points p0L [3][51]."""
    synth = importlib.import_module("3di_b200.synth")
    ex, ey, ez, slo, sup = BASES[cfg["EXP_BASIS"]]
    EX, EY, EZ = (read_matrix(os.path.join(model_dir, f)) for f in (ex, ey, ez))
    V, K = EX.shape
    ident = read_matrix(shp, 3)
    albedo = read_matrix(tex, 1)[:, 0]
    if ident.shape[0] != V or albedo.shape[0] != V:
        raise ValueError(f"identity files have {ident.shape[0]} / {albedo.shape[0]} rows, the model {V}")
    tl = read_matrix(os.path.join(model_dir, "tl.dat"), 3).astype(np.int64) - 1
    lis = read_matrix(os.path.join(model_dir, "li.dat"), 1)[:, 0].astype(np.int32)
    p0L = read_matrix(os.path.join(model_dir, "p0L_mat.dat"), 3).T
    lo = read_matrix(os.path.join(model_dir, slo), 1)[:, 0]
    up = read_matrix(os.path.join(model_dir, sup), 1)[:, 0]
    d, ft = cfg["OPTS_DELTA_EPS"], cfg["FINETUNE_COEF"]
    m = synth.Model(mean=np.ascontiguousarray(ident.T, F32),
                    E=np.ascontiguousarray(np.stack([EX, EY, EZ], axis=1), F32),
                    tex=albedo.astype(F32), tl=np.ascontiguousarray(tl.T, np.int32), lis=lis,
                    eps_lb=(lo * F32(d)).astype(F32), eps_ub=(up * F32(d)).astype(F32),
                    eps_lb_ft=(lo * F32(ft * d)).astype(F32), eps_ub_ft=(up * F32(ft * d)).astype(F32))
    return m, np.ascontiguousarray(p0L, F32)


def read_landmarks(path: str):
    """x, y [T][51] from the interleaved landmark rows (LandmarkData::fill_xpypvec)."""
    a = read_matrix(path)
    if a.shape[1] < 2 * NL:
        raise ValueError(f"{path}: {a.shape[1]} columns, expected {2 * NL}")
    return a[:, 0:2 * NL:2].astype(F32), a[:, 1:2 * NL:2].astype(F32)


def face_size(xp, yp) -> float:
    """LandmarkData::get_face_size (input_data.cu:123-138): integer box extents."""
    w = int(float(np.max(xp))) - int(float(np.min(xp)))
    h = int(float(np.max(yp))) - int(float(np.min(yp)))
    return float(max(w, h))


def camera(arg: str, width: int, height: int) -> np.ndarray:
    """(phix, phiy, cx, cy) from a field of view in degrees or a calibration file."""
    try:
        fov = float(arg)
    except ValueError:
        import cv2
        fs = cv2.FileStorage(arg, cv2.FILE_STORAGE_READ)
        Km = fs.getNode("cameraMatrix_postUndistort").mat()
        fs.release()
        if Km is None:
            raise ValueError(f"{arg}: no cameraMatrix_postUndistort")
        return np.array([Km[0, 0], Km[1, 1], Km[0, 2], Km[1, 2]], F32)
    cx, cy = F32(width / 2.0), F32(height / 2.0)
    ax = F32(float(cx) / math.tan(fov * math.pi / 180.0 / 2.0))
    return np.array([ax, ax, cx, cy], F32)


def constant_bounds(n: int) -> np.ndarray:
    """[n][4][51] landmark boxes lx, ly, ux, uy in face sizes: +-BOX widened by the margin."""
    lo = F32(-BOX) - F32(BOX_MARGIN) * F32(2 * BOX)
    hi = F32(BOX) + F32(BOX_MARGIN) * F32(2 * BOX)
    b = np.empty((n, 4, NL), F32)
    b[:, 0] = lo
    b[:, 1] = lo
    b[:, 2] = hi
    b[:, 3] = hi
    return b


def fit_config(cfg: dict):
    tdi = importlib.import_module("3di_b200")
    return tdi.default_config(max_iters_rigid=100, max_iters_finetune=100, twostage_illum=int(cfg["TWOSTAGE_ILLUM"]),
                              finetune=int(cfg["FINETUNE_EXPRESSIONS"]), niters_success=int(cfg["NITERS_SUCCESS"]),
                              ref_face_size=float(cfg["REF_FACE_SIZE"]), kernel_sigma=float(cfg["KERNEL_SIGMA"]))


class ChunkFitter:
    """Fits chunks of video frames: the landmark check at scale 1, then every reference size of
    every frame of the chunk as one batch (crops, landmark initialisation, image fit)."""

    def __init__(self, m, p0L, cfg: dict, chunk: int):
        tdi = importlib.import_module("3di_b200")
        video = importlib.import_module("3di_b200.video")
        self.K = m.n_expr
        self.p0L = p0L
        self.sizes = [s for s in video.ref_sizes(cfg["REF_FACE_SIZE"], int(cfg["NRES_COEFS"])) if s > 0]
        self.cfg = fit_config(cfg)
        self.model = tdi.Model(m)
        self.check = tdi.Batch(self.model, chunk)
        self.batch = tdi.Batch(self.model, chunk * len(self.sizes))

    def fit(self, bgr, xp, yp, cam, frame_ids, out) -> int:
        """Adds the chunk's reconstructions to out (a VideoOutput); returns how many frames
        passed the landmark check."""
        T = len(frame_ids)
        fs = np.array([face_size(xp[t], yp[t]) for t in range(T)], F32)
        cams = np.tile(cam, (T, 1))
        bounds = constant_bounds(T)
        # the landmark fit on the original frame (scale 1) must succeed (video_fitter.cu:215-270)
        self.check.set_video_frames(bgr, xp, yp, bounds, fs, cams, fs)
        ok, _, _ = self.check.landmark_init(self.p0L)
        keep = np.nonzero(ok)[0]
        if len(keep) == 0:
            return 0
        S, n = len(self.sizes), len(keep)
        rep = lambda a: np.concatenate([np.asarray(a)[keep]] * S)
        refs = np.repeat(np.asarray(self.sizes, F32), n)
        self.batch.set_video_frames(rep(bgr), rep(xp), rep(yp), rep(bounds), rep(fs), rep(cams), refs)
        self.batch.landmark_init(self.p0L)
        self.batch.set_state(None, np.tile(LAMBDA0, (S * n, 1)), np.full(S * n, L0, F32))
        self.batch.fit(self.cfg)
        x, lam, _ = self.batch.get_state()
        for j, t in enumerate(keep):          # per frame, scale by scale (update_shape_single_ref_size)
            for s in range(S):
                f = s * n + j
                out.add_exp_coeffs(frame_ids[t], x[f, :self.K])
                out.add_pose(frame_ids[t], x[f, self.K:self.K + 6])
                out.add_illum(frame_ids[t], np.concatenate([lam[f], [L0]]).astype(F32))
        return n


def fit_video(video_path: str, xps, yps, cam_arg: str, m, p0L, cfg: dict, chunk: int = 64):
    """VideoFitter::fit_video_frames_auto for a window of one frame (video_fitter.cu:116-300):
    returns the VideoOutput of the video's frames."""
    import cv2
    video = importlib.import_module("3di_b200.video")
    cap = cv2.VideoCapture(video_path)
    if not cap.isOpened():
        raise FileNotFoundError(video_path)
    W, H = int(cap.get(cv2.CAP_PROP_FRAME_WIDTH)), int(cap.get(cv2.CAP_PROP_FRAME_HEIGHT))
    fps = cap.get(cv2.CAP_PROP_FPS) or 30.0
    nframes = min(int(cap.get(cv2.CAP_PROP_FRAME_COUNT)), int(cfg["MAX_VID_FRAMES_TO_PROCESS"]), len(xps))
    cam = camera(cam_arg, W, H)
    out = video.VideoOutput(m.n_expr, int(cfg["NRES_COEFS"]))
    fitter = ChunkFitter(m, p0L, cfg, chunk)
    frames, ids = [], []

    def flush():
        if frames:
            idx = np.asarray(ids)
            fitter.fit(np.stack(frames), xps[idx], yps[idx], cam, list(ids), out)
            frames.clear()
            ids.clear()

    for fi in range(nframes):
        ok, frame = cap.read()
        if fi < fps * float(cfg["SKIP_FIRST_N_SECS"]):
            continue
        if not ok:
            break
        xp, yp = xps[fi], yps[fi]
        # landmarks inside the frame (video_fitter.cu:181-190); other frames stay NaN rows
        if not (xp.min() > 0 and yp.min() > 0 and xp.max() < frame.shape[1] and yp.max() < frame.shape[0]):
            continue
        frames.append(frame)
        ids.append(fi)
        if len(frames) == chunk:
            flush()
    flush()
    cap.release()
    return out


def save(out, exp_path: str, pose_path: str, illum_path: str) -> None:
    if not out.abs_frame_ids:
        for p in (exp_path, pose_path, illum_path):
            open(p, "w").close()
        return
    out.save_expressions(exp_path)
    out.save_poses(pose_path)
    out.save_illums(illum_path)


def parse_args(argv):
    ap = argparse.ArgumentParser(prog="video_from_saved_identity",
                                 description="3DMM fit of every video frame with a saved identity (3DI drop-in)")
    for name in ("video", "landmarks", "config", "camera", "shp", "tex", "out_expressions", "out_poses",
                 "out_illums"):
        ap.add_argument(name)
    ap.add_argument("--models-root", default=".", help="directory holding models/MMs/<MM>/ (default: .)")
    ap.add_argument("--chunk", type=int, default=64, help="video frames fitted together (x NRES_COEFS fits)")
    return ap.parse_args(argv)


def main(argv=None) -> int:
    a = parse_args(sys.argv[1:] if argv is None else argv)
    tdi = importlib.import_module("3di_b200")
    tdi.require_gpu()
    cfg = read_config(a.config)
    model_dir = os.path.join(a.models_root, "models", "MMs", cfg["MM"])
    m, p0L = read_model(model_dir, cfg, a.shp, a.tex)
    xps, yps = read_landmarks(a.landmarks)
    out = fit_video(a.video, xps, yps, a.camera, m, p0L, cfg, chunk=a.chunk)
    save(out, a.out_expressions, a.out_poses, a.out_illums)
    return 0


if __name__ == "__main__":
    sys.exit(main())
