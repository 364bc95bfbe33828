"""Video output of the batched fit: the reference's multi-scale fitting of a frame window and
the per-frame averages it writes as text.

* ``ref_sizes``: the list of reference face sizes a window is fitted at
  (src/lib/video_fitter.cu:271-280, REF_EXTRA = 5 from :145), truncated or zero-padded to
  NRES_COEFS entries as ``std::vector::resize`` does.
* ``fit_multiscale``: VideoFitter::update_shape_single_ref_size (video_fitter.cu:355-393) for
  every scale, run as ONE batch of (scales x frames) fits: each scale re-forms its crops from
  the raw frames on the device (tdi_batch_set_video_frames with per-frame reference sizes),
  and the results enter the output scale by scale, frame by frame, in the reference's order.
* ``VideoOutput``: the reference's VideoOutput (video_fitter.cu:2603-2830, video_fitter.h:33-60):
  per absolute frame id, every reconstruction's expression coefficients and pose, the first
  illumination; averages in FP32 in insertion order; frames without any reconstruction read as
  NaN rows (the per-frame failure convention); ``save_*`` write the ``.expressions``,
  ``.poses`` and ``.illums`` text files with write_2d_vector's layout (funcs.h:112-124: values
  with 7 significant digits, each followed by a space, one row per line, every row as long as
  the first).

Euler angles in ``save_poses`` follow RotationComputer::compute_euler_angles
(rotation_header.cu:421-449) on R(u) formed on the host with the library's rotation formula;
the reference's own save_poses reads rotations through an out-of-range frame pointer, so
that step is restated rather than reproduced.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32
REF_EXTRA = 5.0


def ref_sizes(ref_face_size: float, nres: int, ref_extra: float = REF_EXTRA) -> list:
    """Reference face sizes of one window, in the reference's order (FP32 sums)."""
    rs, re = F32(ref_face_size), F32(ref_extra)
    re2 = F32(re / F32(2.0))
    offs = [(re, 5.0), (re, 3.0), (re, 9.0), (re, 7.0), (re, -9.0), (re, -6.0), (re, -3.0),
            (re2, 5.0), (re2, 3.0), (re2, 9.0), (re2, 7.0), (re2, -9.0), (re2, -6.0), (re2, -3.0)]
    out = [rs] + [F32(F32(rs + e) + F32(d)) for e, d in offs]
    out = out[:nres] + [F32(0.0)] * max(0, nres - len(out))
    return out


def rotation_matrix(u) -> np.ndarray:
    """R(u) with the library's FP32 operation order (column-major 3x3, as the kernels store it)."""
    u = [F32(v) for v in u]
    theta = F32(math.sqrt(float(F32(F32(u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]))))
    un = [F32(v / theta) for v in u]

    def skew(w):
        return [F32(0), w[2], F32(-w[1]), F32(-w[2]), F32(0), w[0], w[1], F32(-w[0]), F32(0)]

    def mul33(A, B):
        C = [F32(0)] * 9
        for col in range(3):
            for row in range(3):
                C[3 * col + row] = F32(F32(F32(A[row] * B[3 * col]) + F32(A[3 + row] * B[3 * col + 1]))
                                       + F32(A[6 + row] * B[3 * col + 2]))
        return C

    Sn = skew(un)
    Sn2 = mul33(Sn, Sn)
    st = F32(math.sin(float(theta)))
    cis = F32(F32(1.0) - F32(math.cos(float(theta))))
    R = []
    for i in range(9):
        v = F32(cis * Sn2[i])
        if i in (0, 4, 8):
            v = F32(v + F32(1.0))
        R.append(F32(v + F32(st * Sn[i])))
    return np.array(R, F32)


def euler_angles(R) -> tuple:
    """(yaw, pitch, roll) of a column-major rotation (rotation_header.cu:421-449)."""
    R = [F32(v) for v in R]
    c = F32(math.sqrt(float(F32(F32(R[5] * R[5]) + F32(R[8] * R[8])))))
    if not c < F32(1e-6):
        roll = F32(math.atan2(float(R[1]), float(R[0])))
        yaw = F32(math.atan2(float(-R[2]), float(c)))
        pitch = F32(math.atan2(float(R[5]), float(R[8])))
    else:
        roll = F32(math.atan2(float(-R[7]), float(R[4])))
        yaw = F32(math.atan2(float(-R[2]), float(c)))
        pitch = F32(0.0)
    return yaw, pitch, roll


def write_2d_vector(path: str, rows) -> None:
    """funcs.h:112-124: '%.7g ' per value (the first row's length for every row), '\\n' per row."""
    with open(path, "w") as fh:
        if not rows:
            return
        n = len(rows[0])
        for r in rows:
            fh.write("".join("%.7g " % float(F32(r[j])) for j in range(n)) + "\n")


class VideoOutput:
    """Per-frame results of the reconstructions of a video (video_fitter.cu:2603-2830)."""

    def __init__(self, K: int, nres: int = 4):
        self.K = K
        self.nres = nres
        self.exp_coefs: dict[int, list] = {}
        self.poses: dict[int, list] = {}
        self.illums: dict[int, np.ndarray] = {}
        self.abs_frame_ids: set[int] = set()

    def add_exp_coeffs(self, frame_id: int, coefs) -> None:
        self.exp_coefs.setdefault(int(frame_id), []).append(np.asarray(coefs, F32).copy())
        self.abs_frame_ids.add(int(frame_id))

    def add_pose(self, frame_id: int, pose) -> None:
        self.poses.setdefault(int(frame_id), []).append(np.asarray(pose, F32).copy())

    def add_illum(self, frame_id: int, illum) -> None:
        self.illums.setdefault(int(frame_id), np.asarray(illum, F32).copy())   # the first one stays

    def compute_avg_exp_coeffs(self, frame_id: int, ignore_first: bool = False) -> np.ndarray:
        if frame_id not in self.exp_coefs:
            return np.full(self.K, np.nan, F32)
        rec = self.exp_coefs[frame_id]
        k0 = 1 if ignore_first else 0
        avg = np.zeros(self.K, F32)
        with np.errstate(divide="ignore", invalid="ignore"):
            n = F32(len(rec) - k0)
            for k in range(k0, len(rec)):
                avg = (avg + (rec[k] / n).astype(F32)).astype(F32)
        return avg

    def combine_exp_coeffs(self, frame_id: int) -> np.ndarray:
        out = np.full(self.K * self.nres, np.nan, F32)
        for k, c in enumerate(self.exp_coefs.get(frame_id, [])[:self.nres]):
            out[k * self.K:(k + 1) * self.K] = c
        return out

    def compute_avg_pose(self, frame_id: int) -> np.ndarray:
        if frame_id not in self.poses:
            return np.full(6, np.nan, F32)
        rec = self.poses[frame_id]
        n = F32(len(rec))
        avg = np.zeros(6, F32)
        for p in rec:
            avg = (avg + (p / n).astype(F32)).astype(F32)
        return avg

    def get_illum(self, frame_id: int) -> np.ndarray:
        return self.illums.get(frame_id, np.full(4, np.nan, F32)).copy()

    def compute_avg_illum_last_k_frames(self, cur_frame_id: int, K: int) -> np.ndarray:
        out = np.zeros(4, F32)
        n = 0
        for t in range(max(0, cur_frame_id - K), cur_frame_id):
            c = self.get_illum(t)
            if not np.isnan(c[0]):
                n += 1
                out = (out + c).astype(F32)
        if n > 0:
            out = (out / F32(n)).astype(F32)
        return out

    def _max_id(self) -> int:
        return max(self.abs_frame_ids)

    def save_expressions(self, path: str, ignore_first: bool = False) -> None:
        # frames 0 .. max id - 1, as the reference writes them
        write_2d_vector(path, [self.compute_avg_exp_coeffs(t, ignore_first) for t in range(self._max_id())])

    def save_expressions_all(self, path: str) -> None:
        write_2d_vector(path, [self.combine_exp_coeffs(t) for t in range(self._max_id() + 1)])

    def save_poses(self, path: str, with_angles: bool = True) -> None:
        rows = []
        for t in range(self._max_id()):
            p = list(self.compute_avg_pose(t))
            if with_angles:
                p += list(euler_angles(rotation_matrix(p[3:6])))
            rows.append(p)
        write_2d_vector(path, rows)

    def save_illums(self, path: str) -> None:
        write_2d_vector(path, [self.get_illum(t) for t in range(self._max_id())])


def fit_multiscale(batch, bgr, xp, yp, bounds, face_size, cam, x0, lam0, L, cfg, sizes, frame_ids,
                   out: VideoOutput):
    """Fits a window of T frames at every reference size in one batch of len(sizes) * T fits
    and adds the results to ``out`` as update_shape_single_ref_size does (scale by scale,
    frame by frame). x0, lam0: [T][...] (every scale starts from the same state) or
    [S][T][...]. Returns the reports, [S][T]."""
    S, T = len(sizes), len(frame_ids)
    K = batch.model.K

    def per_scale(a):          # [T][n] for every scale, or [S][T][n]
        a = np.asarray(a, F32)
        return a.reshape(S * T, a.shape[2]) if a.ndim == 3 else np.concatenate([a] * S)

    def rep_(a):               # the same frames for every scale
        return np.concatenate([np.asarray(a)] * S)

    refs = np.repeat(np.asarray(sizes, F32), T)
    batch.set_video_frames(rep_(bgr), rep_(xp), rep_(yp), rep_(bounds), rep_(face_size), rep_(cam), refs)
    x0s, lam0s, Ls = per_scale(x0), per_scale(lam0), rep_(np.asarray(L, F32))
    batch.set_state(x0s, lam0s, Ls)
    batch.fit(cfg)
    x, lam, rep = batch.get_state()
    for s in range(S):
        for t in range(T):
            f = s * T + t
            out.add_exp_coeffs(frame_ids[t], x[f, :K])
            out.add_pose(frame_ids[t], x[f, K:K + 6])
            out.add_illum(frame_ids[t], np.concatenate([lam[f], Ls[f:f + 1]]))
    return [[rep[s * T + t] for t in range(T)] for s in range(S)]
