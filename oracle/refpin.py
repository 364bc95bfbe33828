"""ctypes front end of the reference's own kernels (oracle/_ref/). TEST INFRASTRUCTURE ONLY.

3DI's hot-path CUDA sources (src/lib/funcs.cu, newfuncs.cu, rotation_header.cu) are compiled
unmodified by ``oracle/ref.mk`` together with a driver of this project (``ref_harness.cu``)
into two libraries: ``libtdi_ref_nofma.so`` (no FMA contraction, the oracle's arithmetic
contract) and ``libtdi_ref.so`` (nvcc's default flags, as the reference's own CMake build
compiles them). Tests use them to pin the CPU oracle to the reference: the same inputs go to
both, and the outputs are compared. Needs a GPU; nothing in the product loads these libraries.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_SOURCES = "/root/reference/src/lib"
NPIX = 65536
_LIBS: dict[bool, C.CDLL] = {}


def lib_path(nofma: bool = True) -> str:
    return os.path.join(REF_DIR, "libtdi_ref_nofma.so" if nofma else "libtdi_ref.so")


def available() -> bool:
    return os.path.exists(lib_path(True)) and os.path.exists(lib_path(False))


def build() -> bool:
    """Builds oracle/_ref/ from the reference checkout when it is present; returns whether the
    libraries exist afterwards."""
    if os.path.isdir(REF_SOURCES):
        subprocess.run(["make", "-s", "-f", "ref.mk", "-C", HERE], check=True)
    return available()


def _lib(nofma: bool) -> C.CDLL:
    if nofma not in _LIBS:
        L = C.CDLL(lib_path(nofma))
        vp, ip, fp = C.c_void_p, C.c_int, C.c_float
        L.ref_create.restype = vp
        L.ref_create.argtypes = [ip, ip, ip, vp, vp, vp, vp]
        L.ref_destroy.argtypes = [vp]
        L.ref_rotation.argtypes = [vp, vp, vp, vp]
        L.ref_view_transform.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        L.ref_raster.argtypes = [vp, vp, vp, vp, ip, ip, vp, vp, vp, vp, vp, ip]
        L.ref_evaluate.argtypes = [vp, vp, vp, vp, vp, vp, fp, vp, vp, ip, ip, fp, ip] + [vp] * 12
        _LIBS[nofma] = L
    return _LIBS[nofma]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class RefSession:
    """The reference's kernels on one model (a synth.Model): buffers persist between calls,
    as the reference's Renderer and Optimizer buffers do."""

    def __init__(self, m, taps, nofma: bool = True):
        self.L = _lib(nofma)
        self.V, self.T, self.K = m.n_vertices, m.n_triangles, m.n_expr
        self._tl = np.ascontiguousarray(m.tl, dtype=np.int32)
        self._E = _f32(m.E)
        self._tex = _f32(m.tex)
        self._taps = _f32(taps)
        h = self.L.ref_create(self.V, self.T, self.K, _p(self._tl), _p(self._E), _p(self._tex), _p(self._taps))
        if not h:
            raise RuntimeError("ref_create failed (model beyond 16-bit indices, or a CUDA error)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rotation(self, u):
        R = np.zeros(9, np.float32)
        dR = np.zeros(27, np.float32)
        assert self.L.ref_rotation(self.h, _p(_f32(u)), _p(R), _p(dR)) == 0
        return R, dR.reshape(3, 9)

    def view_transform(self, X0, Y0, Z0, R, tau, cam):
        out = np.zeros((5, self.V), np.float32)
        st = self.L.ref_view_transform(self.h, _p(_f32(X0)), _p(_f32(Y0)), _p(_f32(Z0)), _p(_f32(R)),
                                       _p(_f32(tau)), _p(_f32(cam)), _p(out))
        assert st == 0
        return out

    def raster(self, xp, yp, Z, x0, y0):
        cap = 4 * self.T
        o = dict(pix=np.zeros(cap, np.int32), tri=np.zeros(cap, np.int32), al=np.zeros(cap, np.float32),
                 be=np.zeros(cap, np.float32), ga=np.zeros(cap, np.float32))
        N = self.L.ref_raster(self.h, _p(_f32(xp)), _p(_f32(yp)), _p(_f32(Z)), int(x0), int(y0),
                              _p(o["pix"]), _p(o["tri"]), _p(o["al"]), _p(o["be"]), _p(o["ga"]), cap)
        if N < 0:
            raise RuntimeError(f"ref_raster returned {N}")
        out = {k: v[:N].copy() for k, v in o.items()}
        out["pix"] = out["pix"].astype(np.uint16)
        out["N"] = N
        return out

    def evaluate(self, geo, R, dR, tau, lam, L, cam, target, x0, y0, tau_img=25.0):
        """One image-term evaluation (render, Jacobian rows, chain rule, cuBLAS products)."""
        cap = min(4 * self.T, 25600)
        KT = self.K + 6
        o = dict(pix=np.zeros(cap, np.int32), tri=np.zeros(cap, np.int32), al=np.zeros(cap, np.float32),
                 be=np.zeros(cap, np.float32), shade=np.zeros(cap, np.float32), image=np.zeros(NPIX, np.float32),
                 grads=np.zeros(7 * cap, np.float32), nb=np.zeros(4 * cap, np.int32),
                 J=np.zeros(cap * KT, np.float32), H=np.zeros(KT * KT, np.float32), g=np.zeros(KT, np.float32),
                 corr=np.zeros(1, np.float32))
        N = self.L.ref_evaluate(self.h, _p(_f32(geo)), _p(_f32(R)), _p(_f32(dR)), _p(_f32(tau)), _p(_f32(lam)),
                                float(L), _p(_f32(cam)), _p(_f32(target)), int(x0), int(y0), float(tau_img), cap,
                                *[_p(o[k]) for k in ("pix", "tri", "al", "be", "shade", "image", "grads", "nb",
                                                     "J", "H", "g", "corr")])
        if N < 0:
            raise RuntimeError(f"ref_evaluate returned {N}")
        return dict(N=N, pix=o["pix"][:N].astype(np.uint16), tri=o["tri"][:N].copy(), al=o["al"][:N].copy(),
                    be=o["be"][:N].copy(), shade=o["shade"][:N].copy(), image=o["image"],
                    grads=o["grads"][:7 * N].reshape(7, N).copy(), nb=o["nb"][:4 * N].reshape(4, N).copy(),
                    J=o["J"][:N * KT].reshape(N, KT).copy(),
                    H=o["H"].reshape(KT, KT).T.copy(), g=o["g"].copy(), corr=float(o["corr"][0]))
