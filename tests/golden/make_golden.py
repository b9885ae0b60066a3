"""Generates tests/golden/image_ops.npz: OpenCV's own outputs for the image
stages the reference runs through OpenCV (its GaussianBlur behind cvSmooth,
erode/dilate, medianBlur, cvtColor, remap, perspectiveTransform), used to pin
oracle/image_ops.py.  Needs cv2 (4.13 here); the committed .npz is what the
tests read.

    python tests/golden/make_golden.py
"""
import os

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    rng = np.random.default_rng(20261203)
    H, W = 37, 53
    g = {"cv2_version": np.array(cv2.__version__)}
    img = rng.random((H, W), dtype=np.float32)
    g["img"] = img
    # cvSmooth(CV_GAUSSIAN, 5) = GaussianBlur 5x5, sigma from the size, replicated borders
    g["gauss5"] = cv2.GaussianBlur(img, (5, 5), 0, borderType=cv2.BORDER_REPLICATE)
    u8 = rng.integers(0, 256, (H, W), dtype=np.uint8)
    g["u8"] = u8
    g["median7_u8"] = cv2.medianBlur(u8, 7)
    # Dilate stage: cvErode then cvDilate, 3 iterations, default 3x3 element and border
    disp = (rng.integers(0, 64, (H, W)).astype(np.float32) / np.float32(64.0))
    g["disp_f32"] = disp
    g["open7_f32"] = cv2.dilate(cv2.erode(disp, None, iterations=3), None, iterations=3)
    disp16 = rng.integers(0, 300, (H, W)).astype(np.uint16)
    disp16[rng.random((H, W)) < 0.05] = 0xFFFF
    g["disp_u16"] = disp16
    g["open7_u16"] = cv2.dilate(cv2.erode(disp16, None, iterations=3), None, iterations=3)
    g["median3_f32"] = cv2.medianBlur(disp, 3)
    g["median3_u16"] = cv2.medianBlur(disp16, 3)
    # input conversion: 1/255 scale then RGB2GRAY
    color = rng.integers(0, 256, (H, W, 3), dtype=np.uint8)
    g["color"] = color
    scaled = cv2.multiply(color.astype(np.float32), 1.0 / 255.0)
    g["scaled"] = scaled
    g["gray"] = cv2.cvtColor(scaled, cv2.COLOR_RGB2GRAY)
    # remap, bilinear, constant 0 border, maps reaching outside the source
    mx = (rng.random((H, W), dtype=np.float32) * (W + 6) - 3).astype(np.float32)
    my = (rng.random((H, W), dtype=np.float32) * (H + 6) - 3).astype(np.float32)
    mx[0, :4] = [0.5, 1.0 / 64.0, 3.0 / 64.0, -0.5 / 32.0]  # ties of the 1/32 rounding
    g["mapx"], g["mapy"] = mx, my
    g["remap_f32"] = cv2.remap(img, mx, my, cv2.INTER_LINEAR, borderMode=cv2.BORDER_CONSTANT, borderValue=0)
    g["remap_u8c3"] = cv2.remap(color, mx, my, cv2.INTER_LINEAR, borderMode=cv2.BORDER_CONSTANT, borderValue=0)
    # CVReprojector: perspectiveTransform of (x, H - y, d)
    Q = np.array([[1, 0, 0, -26.5], [0, 1, 0, -18.25], [0, 0, 0, 700.0], [0, 0, -1.0 / 3.5, 0.75]], np.float32)
    g["Q"] = Q
    yy, xx = np.indices((H, W))
    pts = np.stack([xx, H - yy, disp], axis=-1).astype(np.float32).reshape(1, -1, 3)
    g["persp"] = cv2.perspectiveTransform(pts, Q).reshape(H, W, 3)
    # cvInitUndistortRectifyMap with a 5- and an 8-coefficient distortion
    K = np.array([[820.5, 0, 30.2], [0, 815.1, 21.7], [0, 0, 1]])
    R = cv2.Rodrigues(np.array([0.01, -0.02, 0.005]))[0]
    P = np.array([[790.0, 0, 27.5, 0], [0, 790.0, 18.25, 0], [0, 0, 1, 0]])
    g["K"], g["R"], g["P"] = K, R, P
    for name, dist in (("5", [-0.28, 0.09, 0.0012, -0.0007, -0.011]),
                       ("8", [-0.2, 0.05, 0.001, 0.0005, 0.01, 0.02, -0.01, 0.003])):
        mxr, myr = cv2.initUndistortRectifyMap(K, np.array(dist), R, P, (W, H), cv2.CV_32FC1)
        g["dist" + name], g["rmapx" + name], g["rmapy" + name] = np.array(dist), mxr, myr
    np.savez_compressed(os.path.join(HERE, "image_ops.npz"), **g)


if __name__ == "__main__":
    main()
