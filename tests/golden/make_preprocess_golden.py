"""Golden crops for the device preprocessing (tdi_batch_set_video_frames), made with
OpenCV itself: opencv-python 4.13.0 (the reference's image library), Intel IPP switched off
so that cv::resize takes OpenCV's own code (IPP's float resize rounds differently).

Run from the repository root: python tests/golden/make_preprocess_golden.py
Writes tests/golden/preprocess_golden.npz. The reference's steps (input_data.cu:43-53,
video_fitter.cu:537-550):
    cvtColor(frame, gray, COLOR_BGR2GRAY); gray.convertTo(gray, CV_32FC1); gray = gray / 255;
    resize(gray, gray, Size(), c, c); copyMakeBorder(gray, gray, 0, 256, 0, 256, BORDER_CONSTANT, 0);
    crop = gray(Rect(x0, y0, 256, 256)).t()
`gray / 255` is a MatExpr evaluated by convertTo with scale 1/255 (the float scale times
each value); the Python API has no call for that expression, so that one product is
written out here. Landmark rescaling, camera and crop origin follow camera.h:162-174,
input_data.cu:32-40 and renderer.cu:580-598.
"""
import os
import numpy as np
import cv2

HERE = os.path.dirname(os.path.abspath(__file__))
NL, DIM = 51, 256


def crop_origin(xl, yl):
    sz = np.float32(max(np.float32(xl.max() - xl.min()), np.float32(yl.max() - yl.min())))
    x0 = np.float32(float(xl.min()) - float(sz) / 1.5)
    y0 = np.float32(float(yl.min()) - float(sz) / 1.5)
    return int(max(x0, np.float32(0))) & 0xFFFF, int(max(y0, np.float32(0))) & 0xFFFF


def frame(seed, W, H):
    """Smooth shading plus texture and noise, so that resampling errors show."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    base = 128 + 90 * np.sin(xx / 23.0 + seed) * np.cos(yy / 17.0)
    img = np.stack([base + 30 * np.sin(xx / 5.0), base, base - 25 * np.cos(yy / 7.0)], -1)
    img = img + rng.normal(0, 12, img.shape)
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def main():
    assert cv2.__version__ == "4.13.0", cv2.__version__
    cv2.ipp.setUseIPP(False)
    ref_face_size = np.float32(86.0)
    cases = [  # (seed, W, H, face size, landmark box centre)
        (1, 320, 240, 260.0, (170.0, 125.0)),   # downscale 0.331
        (2, 96, 80, 48.0, (50.0, 40.0)),        # upscale 1.79
        (3, 200, 150, 172.0, (100.0, 75.0)),    # exactly half size
        (4, 240, 180, 120.0, (225.0, 170.0)),   # face at the corner: the crop runs into the border
    ]
    out = {}
    for k, (seed, W, H, fs, (cx, cy)) in enumerate(cases):
        bgr = frame(seed, W, H)
        rng = np.random.default_rng(100 + seed)
        xp = (cx + rng.uniform(-0.5, 0.5, NL) * fs).astype(np.float32)
        yp = (cy + rng.uniform(-0.5, 0.5, NL) * fs).astype(np.float32)
        cam = np.array([1000.0, 1000.0, W / 2.0, H / 2.0], np.float32)
        c = np.float32(ref_face_size / np.float32(fs))
        xl, yl = (c * xp).astype(np.float32), (c * yp).astype(np.float32)
        x0, y0 = crop_origin(xl, yl)
        g8 = cv2.cvtColor(bgr, cv2.COLOR_BGR2GRAY)
        g = g8.astype(np.float32) * np.float32(1.0 / 255.0)
        r = cv2.resize(g, None, fx=float(c), fy=float(c), interpolation=cv2.INTER_LINEAR)
        p = cv2.copyMakeBorder(r, 0, DIM, 0, DIM, cv2.BORDER_CONSTANT, value=0)
        big = np.zeros((y0 + DIM, x0 + DIM), np.float32)
        hh, ww = min(p.shape[0], big.shape[0]), min(p.shape[1], big.shape[1])
        big[:hh, :ww] = p[:hh, :ww]
        crop = np.ascontiguousarray(big[y0:y0 + DIM, x0:x0 + DIM].T).reshape(-1)
        out[f"bgr{k}"] = bgr
        out[f"xp{k}"], out[f"yp{k}"] = xp, yp
        out[f"cam{k}"] = cam
        out[f"face_size{k}"] = np.float32(fs)
        out[f"crop{k}"] = crop
        out[f"x0y0_{k}"] = np.array([x0, y0], np.int32)
    out["ref_face_size"] = ref_face_size
    out["n_cases"] = np.int32(len(cases))
    np.savez_compressed(os.path.join(HERE, "preprocess_golden.npz"), **out)


if __name__ == "__main__":
    main()
