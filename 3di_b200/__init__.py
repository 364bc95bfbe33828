"""B200 implementation of 3DI's per-frame 3DMM fitting path.

Python host side over the C ABI of ``libtdi_b200.so`` (declared in ``include/tdi.h``).
The objects mirror the reference's fitting interface: a morphable ``Model`` (the
Renderer's bases, src/lib/renderer.cu:22-442), a ``Batch`` of frames fitted together
(VideoFitter's working set, src/lib/video_fitter.cu:16-81) and ``Batch.fit`` for
VideoFitter::fit_to_video_frame's fitting calls (video_fitter.cu:432-648). Every call goes
to the CUDA library; there is no CPU path, and a missing library or GPU raises.

The package directory name starts with a digit, so import it with
``importlib.import_module("3di_b200")``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtdi_b200.so")
HEADER = os.path.join(HERE, "..", "include", "tdi.h")
NL = 51
NPIX = 65536

FLAG_RENDER_SKIPPED = 1
FLAG_OUT_OF_DOMAIN = 2
FLAG_NAN_DIRECTION = 4
FLAG_STUCK_NEG_TZ = 8
FLAG_CHOL_FAILED = 16
FLAG_FAIL = 32
FLAG_OVERFLOW = 64
FLAG_BAD_INDEX = 128

READ_FRAGMENTS, READ_NEIGHBOURS, READ_GRADIENTS, READ_JACOBIAN, READ_NORMAL_EQ, READ_SCALARS, \
    READ_GEOMETRY, READ_CROP, READ_FRAME_DATA = range(9)


class TdiError(RuntimeError):
    pass


class ModelDesc(C.Structure):
    _fields_ = [("n_vertices", C.c_int32), ("n_triangles", C.c_int32), ("n_expr", C.c_int32),
                ("mean", C.c_void_p), ("expr_basis", C.c_void_p), ("tex", C.c_void_p),
                ("triangles", C.c_void_p), ("landmarks", C.c_void_p),
                ("eps_lb", C.c_void_p), ("eps_ub", C.c_void_p),
                ("eps_lb_finetune", C.c_void_p), ("eps_ub_finetune", C.c_void_p)]


class FramesDesc(C.Structure):
    _fields_ = [("n_frames", C.c_int32), ("targets", C.c_void_p), ("xl", C.c_void_p),
                ("yl", C.c_void_p), ("bounds", C.c_void_p), ("face_size", C.c_void_p),
                ("cam", C.c_void_p), ("x0y0", C.c_void_p)]


class VideoFramesDesc(C.Structure):
    _fields_ = [("n_frames", C.c_int32), ("width", C.c_int32), ("height", C.c_int32),
                ("row_bytes", C.c_int64), ("bgr", C.c_void_p), ("xp", C.c_void_p), ("yp", C.c_void_p),
                ("bounds", C.c_void_p), ("face_size", C.c_void_p), ("cam", C.c_void_p),
                ("ref_face_size", C.c_float), ("ref_face_sizes", C.c_void_p)]


class FitConfig(C.Structure):
    _fields_ = [("max_iters_rigid", C.c_int32), ("max_iters_finetune", C.c_int32),
                ("twostage_illum", C.c_int32), ("finetune", C.c_int32),
                ("niters_success", C.c_int32), ("max_iters_lambda", C.c_int32),
                ("ref_face_size", C.c_float), ("taps", C.c_float * 15), ("normal_eq", C.c_int32),
                ("damping", C.c_float), ("host_rounds", C.c_int32), ("vertex_stage", C.c_int32)]


class Report(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("n_fragments", C.c_int32), ("iters_rigid", C.c_int32),
                ("iters_finetune", C.c_int32), ("iters_lambda", C.c_int32),
                ("renders", C.c_int32), ("objective", C.c_float)]


# Every entry point of include/tdi.h with its ctypes signature.
SIGNATURES = {
    "tdi_last_error": (C.c_char_p, []),
    "tdi_model_create": (C.c_int32, [C.POINTER(ModelDesc), C.POINTER(C.c_void_p)]),
    "tdi_model_destroy": (C.c_int32, [C.c_void_p]),
    "tdi_batch_create": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "tdi_batch_destroy": (C.c_int32, [C.c_void_p]),
    "tdi_batch_set_frames": (C.c_int32, [C.c_void_p, C.POINTER(FramesDesc), C.c_void_p]),
    "tdi_batch_set_video_frames": (C.c_int32, [C.c_void_p, C.POINTER(VideoFramesDesc), C.c_void_p]),
    "tdi_orthographic_init": (C.c_int32, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdi_apply_identity": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32] + [C.c_void_p] * 9),
    "tdi_batch_set_state": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdi_batch_landmark_init": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdi_batch_loss": (C.c_int32, [C.c_void_p, C.POINTER(FitConfig), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
    "tdi_batch_loss_backward": (C.c_int32, [C.c_void_p, C.POINTER(FitConfig), C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdi_batch_fit": (C.c_int32, [C.c_void_p, C.POINTER(FitConfig), C.c_void_p]),
    "tdi_batch_get_state": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdi_fit_frames": (C.c_int32, [C.c_void_p, C.POINTER(FramesDesc), C.POINTER(FitConfig),
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdi_batch_evaluate": (C.c_int32, [C.c_void_p, C.POINTER(FitConfig), C.c_int32, C.c_void_p]),
    "tdi_batch_read": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64,
                                   C.POINTER(C.c_int64)]),
    "tdi_batch_raster": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_uint32)]),
    "tdi_batch_render": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdi_batch_launches": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "tdi_batch_profile": (C.c_int32, [C.c_void_p, C.c_int32]),
    "tdi_batch_profile_read": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                           C.POINTER(C.c_int64)]),
    "tdi_raster_noalloc": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
}

KERNEL_IDS = dict(vertex=1, raster=2, render=3, neighbours=4, jacobian=5, normal_eq=6, barrier=7,
                  solve=8, raster_resolve=9)

_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads the CUDA library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise TdiError(f"{path} is missing: run __graft_entry__.build() (nvcc, sm_100a)")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _check(status: int) -> None:
    if status != 0:
        msg = load_library().tdi_last_error().decode(errors="replace")
        raise TdiError(f"tdi status {status}: {msg}")


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def require_gpu() -> None:
    import torch
    if not torch.cuda.is_available():
        raise TdiError("no CUDA device: the fitting path runs only on the GPU")


NORMAL_EQ_EXACT, NORMAL_EQ_TENSOR = 0, 1
VERTEX_EXACT, VERTEX_TENSOR = 0, 1


def default_config(max_iters_rigid=100, max_iters_finetune=100, twostage_illum=0, finetune=0,
                   niters_success=6, max_iters_lambda=10000, ref_face_size=78.0,
                   kernel_sigma=0.75, normal_eq=NORMAL_EQ_EXACT, damping=0.0, host_rounds=0,
                   vertex_stage=VERTEX_EXACT) -> FitConfig:
    """Configuration keys of the reference's YAML config (src/lib/config.cu:350-541), plus
    ``normal_eq``: NORMAL_EQ_EXACT (FP64 in the oracle's order) or NORMAL_EQ_TENSOR
    (split-BF16 products on the tensor cores), and ``damping``: the lambda of the damped
    shape solve (H + lambda I) d = -g; 0 is the reference's undamped solve; ``host_rounds``: 1
    launches every fitting round from the host instead of replaying CUDA graphs of rounds;
    ``vertex_stage``: VERTEX_EXACT (FP32 fused multiply-add chains in the oracle's order) or
    VERTEX_TENSOR (split-BF16 basis products on the tensor cores, FP32 accumulation)."""
    from . import synth
    c = FitConfig(max_iters_rigid, max_iters_finetune, twostage_illum, finetune, niters_success,
                  max_iters_lambda, ref_face_size)
    c.normal_eq = normal_eq
    c.damping = float(damping)
    c.host_rounds = int(host_rounds)
    c.vertex_stage = int(vertex_stage)
    for i, t in enumerate(synth.KERNEL_SIGMA_TAPS[kernel_sigma]):
        c.taps[i] = t
    return c


class Model:
    """Morphable model on the current GPU (identity applied)."""

    def __init__(self, m):
        self._keep = dict(mean=_f32(m.mean), E=_f32(m.E), tex=_f32(m.tex),
                          tl=np.ascontiguousarray(m.tl, dtype=np.int32),
                          lis=np.ascontiguousarray(m.lis, dtype=np.int32),
                          lb=_f32(m.eps_lb), ub=_f32(m.eps_ub), lbf=_f32(m.eps_lb_ft),
                          ubf=_f32(m.eps_ub_ft))
        k = self._keep
        self.V, self.T, self.K = k["mean"].shape[1], k["tl"].shape[1], k["E"].shape[2]
        desc = ModelDesc(self.V, self.T, self.K, *[k[n].ctypes.data for n in
                                                   ("mean", "E", "tex", "tl", "lis", "lb", "ub", "lbf", "ubf")])
        h = C.c_void_p()
        _check(load_library().tdi_model_create(C.byref(desc), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            load_library().tdi_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def apply_identity(mean0, id_basis, alpha, tex0, tex_basis, beta):
    """The subject's shape and albedo (tdi_apply_identity): mean0 [3][V] + id_basis [3][V][Ka] .
    alpha, tex0 [V] + tex_basis [V][Kb] . beta, on the device. Returns (mean [3][V], tex [V])."""
    mean0, tex0 = _f32(mean0), _f32(tex0)
    V = mean0.shape[1]
    KA = 0 if id_basis is None else int(np.shape(id_basis)[2])
    KB = 0 if tex_basis is None else int(np.shape(tex_basis)[1])
    I = _f32(id_basis) if KA else None
    a = _f32(alpha) if KA else None
    T = _f32(tex_basis) if KB else None
    bt = _f32(beta) if KB else None
    mean = np.zeros((3, V), np.float32)
    tex = np.zeros(V, np.float32)
    ptr = lambda x: _p(x) if x is not None else None
    _check(load_library().tdi_apply_identity(V, KA, KB, _p(mean0), ptr(I), ptr(a), _p(tex0), ptr(T), ptr(bt),
                                             _p(mean), _p(tex), None))
    return mean, tex


def orthographic_init(xl, yl, p0L):
    """Orthographic pose initialisation of F frames (tdi_orthographic_init): landmarks xl, yl
    [F][51], the model's landmark points p0L [3][51]. Returns x [F][7] (tau_x, tau_y,
    sigma_x, sigma_y, u1, u2, u3), yaw/pitch/roll in degrees [F][3] and iterations [F]."""
    xl, yl, p0L = _f32(xl), _f32(yl), _f32(p0L)
    F = xl.shape[0]
    x = np.zeros((F, 7), np.float32)
    ypr = np.zeros((F, 3), np.float32)
    it = np.zeros(F, np.int32)
    _check(load_library().tdi_orthographic_init(F, _p(xl), _p(yl), _p(p0L), _p(x), _p(ypr), _p(it), None))
    return x, ypr, it


class Batch:
    """Device working set for up to ``max_frames`` frames fitted together."""

    def __init__(self, model: Model, max_frames: int):
        self.model = model
        self.cap = int(max_frames)
        h = C.c_void_p()
        _check(load_library().tdi_batch_create(model.handle, self.cap, C.byref(h)))
        self.handle = h
        self.n = 0

    def close(self):
        if getattr(self, "handle", None):
            load_library().tdi_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def frames_desc(fr, i0=0, i1=None):
        i1 = fr.n_frames if i1 is None else i1
        keep = dict(t=_f32(fr.target[i0:i1]), xl=_f32(fr.xl[i0:i1]), yl=_f32(fr.yl[i0:i1]),
                    b=_f32(fr.bounds[i0:i1]), fs=_f32(fr.face_size[i0:i1]), cam=_f32(fr.cam[i0:i1]),
                    o=np.ascontiguousarray(fr.x0y0[i0:i1], dtype=np.int32))
        d = FramesDesc(i1 - i0, *[keep[k].ctypes.data for k in ("t", "xl", "yl", "b", "fs", "cam", "o")])
        return d, keep

    def set_frames(self, fr, i0=0, i1=None):
        d, keep = self.frames_desc(fr, i0, i1)
        _check(load_library().tdi_batch_set_frames(self.handle, C.byref(d), None))
        self.n = d.n_frames

    def set_video_frames(self, bgr, xp, yp, bounds, face_size, cam, ref_face_size):
        """Raw frames (the reference's decoded video frames): bgr [F][H][W][3] uint8 (or with a
        row pitch: [F][H][row_bytes]), landmarks xp, yp [F][51] in image pixels, bounds
        [F][4][51], face_size [F] in image pixels, cam [F][4] of the original camera. The
        library rescales each frame by ref_face_size / face_size and forms the crops on the
        device (tdi_batch_set_video_frames)."""
        bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
        F, H = bgr.shape[0], bgr.shape[1]
        row_bytes = int(np.prod(bgr.shape[2:]))
        W = bgr.shape[2] if bgr.ndim == 4 else row_bytes // 3
        xp, yp, bounds, face_size, cam = _f32(xp), _f32(yp), _f32(bounds), _f32(face_size), _f32(cam)
        refs = None
        if np.ndim(ref_face_size) > 0:      # one reference size per frame
            refs = _f32(np.broadcast_to(np.asarray(ref_face_size, np.float32), (F,)))
            ref_face_size = 0.0
        d = VideoFramesDesc(F, W, H, row_bytes, _p(bgr), _p(xp), _p(yp), _p(bounds), _p(face_size),
                            _p(cam), float(ref_face_size), _p(refs) if refs is not None else None)
        _check(load_library().tdi_batch_set_video_frames(self.handle, C.byref(d), None))
        self.n = F

    def set_state(self, x, lam, L):
        """States x [F][K+6] (None keeps the device states), light lam [F][3] and L [F]."""
        lam, L = _f32(lam), _f32(L)
        xp = None
        if x is not None:
            x = _f32(x)
            xp = _p(x)
        _check(load_library().tdi_batch_set_state(self.handle, xp, _p(lam), _p(L), None))

    def landmark_init(self, p0L):
        """Landmark initialisation of the batch's frames (tdi_batch_landmark_init) with the
        orthographic step's landmark points p0L [3][51]. The fitted states stay on the device
        for the image fit; returns per frame (success, slack, Newton iterations)."""
        p0L = _f32(p0L)
        ok = np.zeros(self.n, np.int32)
        slack = np.zeros(self.n, np.float32)
        it = np.zeros(self.n, np.int32)
        _check(load_library().tdi_batch_landmark_init(self.handle, _p(p0L), _p(ok), _p(slack), _p(it), None))
        return ok.astype(bool), slack, it

    def fit(self, cfg: FitConfig, stream=None):
        _check(load_library().tdi_batch_fit(self.handle, C.byref(cfg), stream))

    def get_state(self):
        KT = self.model.K + 6
        x = np.zeros((self.n, KT), np.float32)
        lam = np.zeros((self.n, 3), np.float32)
        rep = (Report * self.n)()
        _check(load_library().tdi_batch_get_state(self.handle, _p(x), _p(lam), rep, None))
        return x, lam, rep

    def fit_frames(self, fr, x, lam, L, cfg: FitConfig):
        """Upload, fit and download in one call (tdi_fit_frames)."""
        d, keep = self.frames_desc(fr)
        x = _f32(x).copy()
        lam = _f32(lam).copy()
        L = _f32(L)
        rep = (Report * d.n_frames)()
        _check(load_library().tdi_fit_frames(self.handle, C.byref(d), C.byref(cfg), _p(x), _p(lam),
                                             _p(L), rep, None))
        self.n = d.n_frames
        return x, lam, rep

    def evaluate(self, cfg: FitConfig, finetune_bounds=False):
        _check(load_library().tdi_batch_evaluate(self.handle, C.byref(cfg), int(finetune_bounds), None))

    def read(self, frame: int, what: int):
        KT = self.model.K + 6
        cap = {READ_FRAGMENTS: 4 * 32768, READ_NEIGHBOURS: 4 * 32768, READ_GRADIENTS: 5 * 32768,
               READ_JACOBIAN: 32768 * KT, READ_NORMAL_EQ: KT * KT + 2 * KT, READ_SCALARS: 4,
               READ_GEOMETRY: 6 * self.model.V, READ_CROP: NPIX, READ_FRAME_DATA: 2 * 51 + 7}[what]
        dt = np.float64 if what == READ_SCALARS else (np.int32 if what in (READ_FRAGMENTS, READ_NEIGHBOURS) else np.float32)
        buf = np.zeros(cap, dt)
        cnt = C.c_int64(0)
        _check(load_library().tdi_batch_read(self.handle, int(frame), int(what), _p(buf),
                                             buf.nbytes, C.byref(cnt)))
        out = buf[:cnt.value]
        if what == READ_FRAGMENTS:
            r = out.reshape(-1, 4)
            pix_owner = r[:, 0].view(np.uint32)
            return dict(pix=(pix_owner & 0xFFFF).astype(np.uint16), owner=(pix_owner >> 31).astype(np.uint8),
                        tri=r[:, 1].copy(), al=r[:, 2].view(np.float32).copy(),
                        be=r[:, 3].view(np.float32).copy())
        if what == READ_NEIGHBOURS:
            return out.reshape(4, -1)
        if what == READ_GRADIENTS:
            return out.reshape(5, -1)
        if what == READ_JACOBIAN:
            return out.reshape(-1, KT)
        if what == READ_NORMAL_EQ:
            return dict(H=out[:KT * KT].reshape(KT, KT), g=out[KT * KT:KT * KT + KT], d=out[KT * KT + KT:])
        if what == READ_SCALARS:
            return dict(corr=out[0], barrier=out[1], objective=out[2], face_ok=bool(out[3]))
        if what == READ_CROP:
            return out.copy()
        if what == READ_FRAME_DATA:
            return dict(xl=out[:51].copy(), yl=out[51:102].copy(), cam=out[102:106].copy(),
                        face_size=float(out[106]), x0=int(out[107]), y0=int(out[108]))
        return out.reshape(6, -1)

    def render(self, want_images=True, want_tri_map=False):
        """Unblurred images and owner-triangle maps of every frame at its current state."""
        img = np.zeros((self.n, NPIX), np.float32) if want_images else None
        tm = np.zeros((self.n, NPIX), np.int32) if want_tri_map else None
        _check(load_library().tdi_batch_render(self.handle, _p(img) if img is not None else None,
                                               _p(tm) if tm is not None else None, None))
        return img, tm

    def launches(self) -> int:
        n = C.c_int64(0)
        _check(load_library().tdi_batch_launches(self.handle, C.byref(n)))
        return n.value

    def profile(self, kernel: str | None):
        _check(load_library().tdi_batch_profile(self.handle, KERNEL_IDS[kernel] if kernel else 0))

    def profile_read(self):
        n, ms, fr = C.c_int64(0), C.c_double(0), C.c_int64(0)
        _check(load_library().tdi_batch_profile_read(self.handle, C.byref(n), C.byref(ms), C.byref(fr)))
        return n.value, ms.value, fr.value

    def raster(self, frame, xp, yp, zc, x0, y0):
        n = C.c_int32(0)
        fl = C.c_uint32(0)
        xp, yp, zc = _f32(xp), _f32(yp), _f32(zc)
        _check(load_library().tdi_batch_raster(self.handle, int(frame), _p(xp), _p(yp), _p(zc),
                                               int(x0), int(y0), C.byref(n), C.byref(fl)))
        return n.value, fl.value


def header_symbols(path: str = HEADER) -> list[str]:
    """Names of the functions include/tdi.h declares."""
    import re
    src = open(path).read()
    return sorted(set(re.findall(r"\b(tdi_[a-z_]+)\s*\(", src)) - {"tdi_status"})
