"""ctypes front end of the CPU oracle (tdi_oracle.c). TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this
module, always as the checker or the timed CPU baseline -- never as part of the product.
3DI ships no golden vectors for this path, so the restatement is pinned to the reference
itself. Its hot-path CUDA sources are built as they lie into ``oracle/_ref/`` (``ref.mk``,
with stand-in headers for the OpenCV display helpers that the path never calls), and
``tests/test_ref_pinning.py`` compares this oracle with them stage by stage on a B200.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NL, NPIX = 51, 65536
_LIBS: dict[str, C.CDLL] = {}

F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OModel(C.Structure):
    _fields_ = [("V", C.c_int32), ("T", C.c_int32), ("K", C.c_int32),
                ("mean", C.c_void_p), ("E", C.c_void_p), ("tex", C.c_void_p),
                ("tl", C.c_void_p), ("lis", C.c_void_p),
                ("eps_lb", C.c_void_p), ("eps_ub", C.c_void_p),
                ("eps_lb_ft", C.c_void_p), ("eps_ub_ft", C.c_void_p)]


class OFrame(C.Structure):
    _fields_ = [("target", C.c_void_p), ("xl", C.c_void_p), ("yl", C.c_void_p),
                ("bounds", C.c_void_p), ("face_size", C.c_float),
                ("phix", C.c_float), ("phiy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("x0", C.c_int32), ("y0", C.c_int32)]


class OConfig(C.Structure):
    _fields_ = [("max_iters_rigid", C.c_int32), ("max_iters_finetune", C.c_int32),
                ("twostage_illum", C.c_int32), ("finetune", C.c_int32),
                ("niters_success", C.c_int32), ("max_iters_lambda", C.c_int32),
                ("ref_face_size", C.c_float), ("taps", C.c_float * 15), ("damping", C.c_float)]


class OReport(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("n_fragments", C.c_int32), ("iters_rigid", C.c_int32),
                ("iters_finetune", C.c_int32), ("iters_lambda", C.c_int32),
                ("renders", C.c_int32), ("objective", C.c_float)]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(kind: str = "f32") -> C.CDLL:
    if kind not in _LIBS:
        path = os.path.join(HERE, f"libtdi_oracle_{kind}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.o_fit_frames.restype = C.c_int
        L.o_evaluate_f.restype = C.c_int
        L.o_raster_f.restype = C.c_int
        L.o_render_image_f.restype = C.c_int
        L.o_vertex_stage_f.restype = C.c_int
        L.o_image_terms_f.restype = C.c_int
        L.o_landmark_init_f.restype = C.c_int
        L.o_max_threads.restype = C.c_int
        _LIBS[kind] = L
    return _LIBS[kind]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Model:
    """Holds contiguous copies of a synth.Model and the o_model struct pointing at them."""

    def __init__(self, m):
        self.mean = _f32(m.mean)
        self.E = _f32(m.E)
        self.tex = _f32(m.tex)
        self.tl = np.ascontiguousarray(m.tl, dtype=np.int32)
        self.lis = np.ascontiguousarray(m.lis, dtype=np.int32)
        self.lb, self.ub = _f32(m.eps_lb), _f32(m.eps_ub)
        self.lb_ft, self.ub_ft = _f32(m.eps_lb_ft), _f32(m.eps_ub_ft)
        self.V, self.T, self.K = self.mean.shape[1], self.tl.shape[1], self.E.shape[2]
        self.s = OModel(self.V, self.T, self.K, _p(self.mean), _p(self.E), _p(self.tex),
                        _p(self.tl), _p(self.lis), _p(self.lb), _p(self.ub),
                        _p(self.lb_ft), _p(self.ub_ft))


class FrameSet:
    """o_frame structs for frames [i0, i1) of a synth.Frames (targets must be present)."""

    def __init__(self, fr, i0=0, i1=None):
        i1 = fr.n_frames if i1 is None else i1
        self.target = _f32(fr.target[i0:i1])
        self.xl, self.yl = _f32(fr.xl[i0:i1]), _f32(fr.yl[i0:i1])
        self.bounds = _f32(fr.bounds[i0:i1])
        n = i1 - i0
        self.arr = (OFrame * n)()
        for j in range(n):
            i = i0 + j
            self.arr[j] = OFrame(_p(self.target[j]), _p(self.xl[j]), _p(self.yl[j]),
                                 _p(self.bounds[j]), float(fr.face_size[i]),
                                 *[float(v) for v in fr.cam[i]],
                                 int(fr.x0y0[i, 0]), int(fr.x0y0[i, 1]))
        self.n = n


def config(max_iters_rigid=100, max_iters_finetune=100, twostage_illum=0, finetune=0,
           niters_success=6, max_iters_lambda=10000, ref_face_size=78.0, taps=None, damping=0.0) -> OConfig:
    if taps is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location(
            "_synth", os.path.join(HERE, "..", "3di_b200", "synth.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        taps = mod.KERNEL_SIGMA_TAPS[0.75]
    c = OConfig(max_iters_rigid, max_iters_finetune, twostage_illum, finetune, niters_success,
                max_iters_lambda, ref_face_size)
    c.damping = float(damping)
    for i, t in enumerate(taps):
        c.taps[i] = t
    return c


def fit_frames(model: Model, frames: FrameSet, cfg: OConfig, x, lam, L, kind="f32", threads=0):
    """Fits every frame (OpenMP over frames). Returns (x, lam, reports)."""
    x = _f32(x).copy()
    lam = _f32(lam).copy()
    L = _f32(L)
    rep = (OReport * frames.n)()
    lib(kind).o_fit_frames(C.byref(model.s), frames.arr, frames.n, C.byref(cfg),
                           _p(x), _p(lam), _p(L), rep, int(threads))
    return x, lam, rep


def evaluate(model: Model, frames: FrameSet, j: int, cfg: OConfig, x, lam, L,
             finetune_bounds=False, kind="f32") -> dict:
    """One full evaluation (render, Jacobian, normal equations, barrier, solve) of frame j."""
    cap = 4 * model.T
    KT = model.K + 6
    o = dict(slot=np.zeros(cap, np.int32), tri=np.zeros(cap, np.int32),
             pix=np.zeros(cap, np.uint16), al=np.zeros(cap, np.float32),
             be=np.zeros(cap, np.float32), ga=np.zeros(cap, np.float32),
             owner=np.zeros(cap, np.uint8), image=np.zeros(NPIX, np.float32),
             sh=np.zeros((14, cap), np.float32), grads=np.zeros((8, cap), np.float32),
             nb=np.zeros((4, cap), np.int32), J=np.zeros((cap, KT), np.float32),
             H=np.zeros((KT, KT), np.float32), g=np.zeros(KT, np.float32),
             d=np.zeros(KT, np.float32), scal=np.zeros(4, np.float64))
    flags = C.c_uint32(0)
    N = lib(kind).o_evaluate_f(
        C.byref(model.s), C.byref(frames.arr[j]), C.byref(cfg), _p(_f32(x)), _p(_f32(lam)),
        C.c_float(float(L)), int(finetune_bounds),
        *[_p(o[k]) for k in ("slot", "tri", "pix", "al", "be", "ga", "owner", "image")],
        _p(o["sh"]), _p(o["grads"]), _p(o["nb"]), _p(o["J"]), _p(o["H"]), _p(o["g"]),
        _p(o["d"]), _p(o["scal"]), C.byref(flags))
    out = {}
    for k in ("slot", "tri", "pix", "al", "be", "ga", "owner"):
        out[k] = o[k][:N].copy()
    out["sh"] = o["sh"].reshape(-1)[:14 * N].reshape(14, N).copy()
    out["grads"] = o["grads"].reshape(-1)[:7 * N].reshape(7, N).copy()
    out["nb"] = o["nb"].reshape(-1)[:4 * N].reshape(4, N).copy()
    out["J"] = o["J"].reshape(-1)[:N * KT].reshape(N, KT).copy()
    out.update(image=o["image"], H=o["H"], g=o["g"], d=o["d"], N=N, flags=flags.value,
               corr=o["scal"][0], barrier=o["scal"][1], objective=o["scal"][2],
               face_ok=bool(o["scal"][3]))
    return out


def image_terms(model: Model, frames: FrameSet, j: int, cfg: OConfig, x, lam, L, tau_img=25.0,
                kind="f32") -> dict:
    """Normal equations of the image term alone (no barrier terms) and the correlation sum."""
    KT = model.K + 6
    H = np.zeros((KT, KT), np.float32)
    g = np.zeros(KT, np.float32)
    corr = C.c_double(0)
    N = lib(kind).o_image_terms_f(C.byref(model.s), C.byref(frames.arr[j]), C.byref(cfg), _p(_f32(x)),
                                  _p(_f32(lam)), C.c_float(float(L)), C.c_float(float(tau_img)), _p(H), _p(g),
                                  C.byref(corr))
    return dict(N=N, H=H, g=g, corr=corr.value)


def raster(model: Model, xp, yp, Z, x0, y0, kind="f32") -> dict:
    cap = 4 * model.T
    o = dict(slot=np.zeros(cap, np.int32), tri=np.zeros(cap, np.int32),
             pix=np.zeros(cap, np.uint16), al=np.zeros(cap, np.float32),
             be=np.zeros(cap, np.float32), ga=np.zeros(cap, np.float32),
             owner=np.zeros(cap, np.uint8))
    flags = C.c_uint32(0)
    N = lib(kind).o_raster_f(C.byref(model.s), _p(_f32(xp)), _p(_f32(yp)), _p(_f32(Z)),
                             int(x0), int(y0), *[_p(o[k]) for k in o], C.byref(flags))
    out = {k: v[:N].copy() for k, v in o.items()}
    out.update(N=N, flags=flags.value)
    return out


def neighbours(pix, kind="f32"):
    pix = np.ascontiguousarray(pix, dtype=np.uint16)
    N = pix.shape[0]
    nb = np.zeros((4, N), np.int32)
    flags = C.c_uint32(0)
    lib(kind).o_neighbours_f(_p(pix), N, _p(nb), C.byref(flags))
    return nb, flags.value


def blur(taps, img, kind="f32"):
    out = np.zeros(NPIX, np.float32)
    lib(kind).o_blur_f(_p(_f32(taps)), _p(_f32(img)), _p(out))
    return out


def rotation(u, kind="f32"):
    R = np.zeros(9, np.float32)
    dR = np.zeros(27, np.float32)
    lib(kind).o_rotation_f(_p(_f32(u)), _p(R), _p(dR))
    return R, dR.reshape(3, 9)


def orthographic(xl, yl, p0L, kind="f32"):
    """Orthographic pose initialisation of one frame: (x [7], rotation of the last trial [9],
    outer iterations)."""
    x = np.zeros(7, np.float32)
    R = np.zeros(9, np.float32)
    q = lib(kind).o_orthographic_f(_p(_f32(xl)), _p(_f32(yl)), _p(_f32(p0L)), _p(x), _p(R))
    return x, R, q


def vertex_stage(model: Model, x, cam, ref_face_size=78.0, kind="f32"):
    geo = np.zeros((8, model.V), np.float32)
    ok = lib(kind).o_vertex_stage_f(C.byref(model.s), _p(_f32(x)), _p(_f32(cam)),
                                    C.c_float(ref_face_size), _p(geo))
    return geo, bool(ok)


def render_target(model: Model, fr, i: int, cfg: OConfig, x, lam, L, kind="f32"):
    """Unblurred render of frame i at state x (the synthetic photo before noise)."""
    tgt = np.zeros(NPIX, np.float32)
    tmp_target = np.zeros(NPIX, np.float32)
    xl, yl = _f32(fr.xl[i]), _f32(fr.yl[i])
    b = _f32(fr.bounds[i])
    f = OFrame(_p(tmp_target), _p(xl), _p(yl), _p(b), float(fr.face_size[i]),
               *[float(v) for v in fr.cam[i]], int(fr.x0y0[i, 0]), int(fr.x0y0[i, 1]))
    flags = C.c_uint32(0)
    N = lib(kind).o_render_image_f(C.byref(model.s), C.byref(f), C.byref(cfg), _p(_f32(x)),
                                   _p(_f32(lam)), C.c_float(float(L)), _p(tgt), C.byref(flags))
    return tgt, N, flags.value


def landmark_init(model: Model, frames: FrameSet, j: int, p0L, kind="f32"):
    """Landmark initialisation of frame j (orthographic step, perspective start, barrier method
    with a slack variable). Returns (x [K+6], slack, success, newton iterations, mirrored)."""
    x = np.zeros(model.K + 6, np.float32)
    slack = C.c_float(0)
    newton = C.c_int(0)
    flip = C.c_int(0)
    ok = lib(kind).o_landmark_init_f(C.byref(model.s), C.byref(frames.arr[j]), _p(_f32(p0L)), _p(x),
                                     C.byref(slack), C.byref(newton), C.byref(flip))
    return x, slack.value, bool(ok), newton.value, bool(flip.value)


def apply_identity(mean0, id_basis, alpha, tex0, tex_basis, beta):
    """The subject's shape and albedo: mean0 + id_basis . alpha, tex0 + tex_basis . beta
    (o_apply_identity; FP32 fused multiply-add chains)."""
    mean0, tex0 = _f32(mean0), _f32(tex0)
    V = mean0.shape[1]
    KA = 0 if id_basis is None else int(np.shape(id_basis)[2])
    KB = 0 if tex_basis is None else int(np.shape(tex_basis)[1])
    I = _f32(id_basis) if KA else np.zeros(1, np.float32)
    a = _f32(alpha) if KA else np.zeros(1, np.float32)
    T = _f32(tex_basis) if KB else np.zeros(1, np.float32)
    b = _f32(beta) if KB else np.zeros(1, np.float32)
    mean = np.zeros((3, V), np.float32)
    tex = np.zeros(V, np.float32)
    lib("f32").o_apply_identity(V, KA, KB, _p(mean0), _p(I), _p(a), _p(tex0), _p(T), _p(b), _p(mean), _p(tex))
    return mean, tex


def solve_shape(H, g, damping=0.0):
    """The shape solve's arithmetic (solve_shape in tdi_oracle.c) restated in numpy float64,
    which rounds every product and difference on its own. The factor is read from the upper
    triangle of H: entry (i, l), i >= l, at H[l, i], with the damping added on the diagonal.
    Pivots have reciprocals r_j = 1 / sqrt(s_j). Each entry's updates L(i,k) L(l,k) are
    subtracted in increasing k. Here they run column by column, which gives each entry the
    same sequence as the C file's dot products. Forward and back substitution take their terms
    in increasing and decreasing k. Returns d = -x as float32, or None when a pivot is not
    positive."""
    Hu = np.triu(np.asarray(H, np.float64))
    A = Hu + np.triu(Hu, 1).T
    n = A.shape[0]
    A[np.arange(n), np.arange(n)] += float(np.float32(damping))
    L = np.zeros((n, n))
    r = np.zeros(n)
    for j in range(n):
        s = A[j, j]
        if not s > 0.0:
            return None
        r[j] = 1.0 / np.sqrt(s)
        c = A[j + 1:, j] * r[j]
        L[j + 1:, j] = c
        A[j + 1:, j + 1:] -= np.outer(c, c)
    t = np.asarray(g, np.float64).copy()
    y = np.zeros(n)
    for k in range(n):
        y[k] = t[k] * r[k]
        t[k + 1:] -= L[k + 1:, k] * y[k]
    t = y.copy()
    for k in range(n - 1, -1, -1):
        y[k] = t[k] * r[k]
        t[:k] -= L[k, :k] * y[k]
    return (-y).astype(np.float32)


def max_threads(kind="f32") -> int:
    return int(lib(kind).o_max_threads())
