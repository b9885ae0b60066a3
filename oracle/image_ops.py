"""CPU restatements of the image stages either side of the matching path --
TEST INFRASTRUCTURE ONLY (imported by tests/ and bench.py's CPU baseline).

numpy, float32 arithmetic in the order the CUDA kernels use, so the kernels
must match bit for bit.  The reference runs these steps through OpenCV (an
unvendored dependency, "2.1 or greater", README:13); the published algorithms
restated here are pinned against OpenCV 4.13's own outputs committed under
tests/golden/ (exact except where noted):

* grey conversion, tdvision/misc.cpp:29-32: cvConvertScale(1/255) then
  CV_RGB2GRAY; channel 0 is weighted as red.  OpenCV sums the three products
  in an order of its own; this restatement sums left to right and stays within
  2 ulp of it.
* rectification maps, tdvision/rectificationcv.cpp:114-117,152-155
  (cvInitUndistortRectifyMap: Brown-Conrady distortion, inverse of P R by
  cofactors, double).  Exact.
* remap, tdvision/rectificationcv.cpp:298-310 (cvRemap, bilinear, constant 0
  border): coordinates rounded to 1/32 pixel, float weights for float images,
  15-bit fixed-point weights with rounding for 8-bit ones.  Exact.
* 5x5 Gaussian, tdvision/medianfiltercpu.cpp:15 (cvSmooth CV_GAUSSIAN 5:
  kernel [1 4 6 4 1]/16, replicated borders), rows then columns in the
  symmetric form c*k2 + (a1+b1)*k1 + (a2+b2)*k0; within 2 ulp of OpenCV.
* 7x7 median, tdvision/medianfilter.cu:37-57 (intended; replicated borders);
  8-bit inputs equal cv2.medianBlur(7).
* opening, tdvision/dilate.cpp:18-19: cvErode then cvDilate, 3 iterations of
  the 3x3 element each = 7x7 minimum then maximum over windows clipped at the
  borders.  Exact.
* 3x3 median, replicated borders.  Exact.
* sub-pixel parabola and reprojection (glreprojection.cpp:30-55,
  directreprojector.hpp:17-20, cvreprojector.cpp:45-60: cvPerspectiveTransform
  in double then z * 24), and the ASCII PLY text of
  tdvision/plymeshexporter.cpp:8-76.
"""
import numpy as np

f32 = np.float32


def scale255():
    """The 1/255 scale of each 8-bit value (double, rounded to float; equal to
    the correctly rounded float quotient for every value)."""
    return (np.arange(256, dtype=np.float64) / 255.0).astype(np.float32)


def to_gray(color):
    t = scale255()[color]
    r, g, b = t[..., 0], t[..., 1], t[..., 2]
    return f32(f32(f32(r * f32(0.299)) + f32(g * f32(0.587))) + f32(b * f32(0.114)))


def remap(src, mapx, mapy):
    """src (H, W) or (H, W, C), uint8 or float32; maps (H', W') float32."""
    src3 = src if src.ndim == 3 else src[..., None]
    Hs, Ws, C = src3.shape
    fx32 = np.clip(mapx.astype(np.float32) * f32(32.0), f32(-1e9), f32(1e9))
    fy32 = np.clip(mapy.astype(np.float32) * f32(32.0), f32(-1e9), f32(1e9))
    X = np.rint(fx32).astype(np.int64)
    Y = np.rint(fy32).astype(np.int64)
    ix, fx = X >> 5, X & 31
    iy, fy = Y >> 5, Y & 31

    def tap(dx, dy):
        xx, yy = ix + dx, iy + dy
        ok = (xx >= 0) & (xx < Ws) & (yy >= 0) & (yy < Hs)
        v = src3[np.clip(yy, 0, Hs - 1), np.clip(xx, 0, Ws - 1)]
        return np.where(ok[..., None], v, 0)

    t00, t01, t10, t11 = tap(0, 0), tap(1, 0), tap(0, 1), tap(1, 1)
    if src.dtype == np.uint8:
        w00 = ((32 - fy) * (32 - fx) * 32)[..., None]
        w01 = ((32 - fy) * fx * 32)[..., None]
        w10 = (fy * (32 - fx) * 32)[..., None]
        w11 = (fy * fx * 32)[..., None]
        acc = t00.astype(np.int64) * w00 + t01 * w01 + t10 * w10 + t11 * w11
        out = np.clip((acc + (1 << 14)) >> 15, 0, 255).astype(np.uint8)
    else:
        ax = (fx.astype(np.float32) * f32(0.03125))[..., None]
        ay = (fy.astype(np.float32) * f32(0.03125))[..., None]
        one = f32(1.0)
        w00, w01 = f32((one - ay) * (one - ax)), f32((one - ay) * ax)
        w10, w11 = f32(ay * (one - ax)), f32(ay * ax)
        s = f32(t00.astype(np.float32) * w00)
        s = f32(s + f32(t01.astype(np.float32) * w01))
        s = f32(s + f32(t10.astype(np.float32) * w10))
        s = f32(s + f32(t11.astype(np.float32) * w11))
        out = s.astype(np.float32)
    return out if src.ndim == 3 else out[..., 0]


def rectify_maps(K, dist, R, P, W, H):
    """cvInitUndistortRectifyMap's model (tdvision/rectificationcv.cpp:114-117,
    152-155), in double: M = P[:, :3] R summed left to right, its inverse by
    cofactors, then per pixel (j, i) the operations in the order the kernel
    rounds them.  dist = (k1, k2, p1, p2, k3, k4, k5, k6), zero-padded."""
    K = np.asarray(K, np.float64).reshape(3, 3)
    R = np.asarray(R, np.float64).reshape(3, 3)
    P = np.asarray(P, np.float64).reshape(3, -1)[:, :3]
    k = np.zeros(8)
    k[:len(dist)] = np.asarray(dist, np.float64)
    k1, k2, p1, p2, k3, k4, k5, k6 = k
    M = np.empty((3, 3))
    for r in range(3):
        for c in range(3):
            M[r, c] = (P[r, 0] * R[0, c] + P[r, 1] * R[1, c]) + P[r, 2] * R[2, c]
    a, b, c, d, e, f, g, h, i = M.ravel()
    A, B, C = e * i - f * h, -(d * i - f * g), d * h - e * g
    det = (a * A + b * B) + c * C
    iR = np.array([[A, -(b * i - c * h), b * f - c * e], [B, a * i - c * g, -(a * f - c * d)],
                   [C, -(a * h - b * g), a * e - b * d]]) / det
    fx, fy, cx, cy = K[0, 0], K[1, 1], K[0, 2], K[1, 2]
    ii, jj = np.indices((H, W)).astype(np.float64)
    lin = [(jj * iR[r, 0] + ii * iR[r, 1]) + iR[r, 2] for r in range(3)]
    w = 1.0 / lin[2]
    x, y = lin[0] * w, lin[1] * w
    x2, y2 = x * x, y * y
    r2 = x2 + y2
    xy2 = (2.0 * x) * y
    kr = (1.0 + ((k3 * r2 + k2) * r2 + k1) * r2) / (1.0 + ((k6 * r2 + k5) * r2 + k4) * r2)
    u = fx * ((x * kr + p1 * xy2) + p2 * (r2 + 2.0 * x2)) + cx
    v = fy * ((y * kr + p1 * (r2 + 2.0 * y2)) + p2 * xy2) + cy
    return u.astype(np.float32), v.astype(np.float32)


def _intensity(img, scale):
    if img.dtype == np.uint8:
        return f32(img.astype(np.float32) * f32(scale))
    return f32(img.astype(np.float32) * f32(scale))


def _sym5(a2, a1, c, b1, b2):
    s = f32(c * f32(0.375))
    s = f32(s + f32(f32(a1 + b1) * f32(0.25)))
    return f32(s + f32(f32(a2 + b2) * f32(0.0625)))


def gauss5(img, scale=1.0):
    a = _intensity(img, scale)
    H, W = a.shape
    P = np.pad(a, 2, mode="edge")
    R = _sym5(P[:, 0:W], P[:, 1:W + 1], P[:, 2:W + 2], P[:, 3:W + 3], P[:, 4:W + 4])
    return _sym5(R[0:H], R[1:H + 1], R[2:H + 2], R[3:H + 3], R[4:H + 4])


def _windows(a, r, mode, fill=None):
    H, W = a.shape
    if mode == "edge":
        P = np.pad(a, r, mode="edge")
    else:
        P = np.pad(a, r, mode="constant", constant_values=fill)
    return np.stack([P[dy:dy + H, dx:dx + W] for dy in range(2 * r + 1) for dx in range(2 * r + 1)])


def median7(img, scale=1.0):
    a = _intensity(img, scale)
    return np.median(_windows(a, 3, "edge"), axis=0).astype(np.float32)


def open7(disp):
    """7x7 minimum then maximum over windows clipped at the borders."""
    if disp.dtype == np.uint16:
        lo, hi = np.uint16(0), np.uint16(0xFFFF)
    else:
        lo, hi = f32(-np.inf), f32(np.inf)
    m = _windows(disp, 3, "const", hi).min(axis=0)
    return _windows(m, 3, "const", lo).max(axis=0).astype(disp.dtype)


def median3(disp):
    return np.median(_windows(disp, 1, "edge"), axis=0).astype(disp.dtype)


def subpixel(S, disp):
    """S (H, W, D) float32, disp (H, W) uint16 -> float32."""
    H, W, D = S.shape
    d = disp.astype(np.int64)
    out = d.astype(np.float32)
    inner = (d > 0) & (d < D - 1)
    dc = np.clip(d, 1, D - 2)
    yy, xx = np.indices((H, W))
    a, b, c = S[yy, xx, dc - 1], S[yy, xx, dc], S[yy, xx, dc + 1]
    den = f32(f32(a + c) - f32(f32(2.0) * b))
    ref = f32(out + f32(f32(a - c) / f32(f32(2.0) * np.where(den > 0, den, f32(1.0)))))
    out = np.where(inner & (den > 0), ref, out)
    return np.where((d == 0xFFFF) | (d >= D), f32(-1.0), out).astype(np.float32)


def reproject(disp, color=None, mode="direct", zscale=1.0, q=None):
    """disp (H, W) float32 or uint16 -> vertices (H, W, 3) float32 and colors
    (H, W, 3) float32 (or None)."""
    H, W = disp.shape
    d = disp.astype(np.float32)
    yy, xx = np.indices((H, W))
    fx = xx.astype(np.float32)
    fy = (H - yy).astype(np.float32)
    if mode == "direct":
        v = np.stack([fx, fy, f32(d * f32(zscale))], axis=-1)
    else:
        Q = np.asarray(q, dtype=np.float32).astype(np.float64).reshape(4, 4)
        X, Y, Z = fx.astype(np.float64), fy.astype(np.float64), d.astype(np.float64)
        rows = [((Q[i, 0] * X + Q[i, 1] * Y) + Q[i, 2] * Z) + Q[i, 3] for i in range(4)]
        w = rows[3]
        ok = np.abs(w) > np.finfo(np.float32).eps
        winv = np.where(ok, 1.0 / np.where(ok, w, 1.0), 0.0)
        v = np.stack([np.where(ok, rows[i] * winv, 0.0).astype(np.float32) for i in range(3)], axis=-1)
        v[..., 2] = f32(v[..., 2] * f32(24.0))
    cols = None
    if color is not None:
        cols = f32(color.astype(np.float32) * f32(np.float32(1.0) / np.float32(255.0)))
    return v.astype(np.float32), cols


def ply_text(vertices, colors=None):
    """The reference's ASCII PLY of a grid mesh (plymeshexporter.cpp:24-73)."""
    H, W = vertices.shape[:2]
    lines = ["ply", "format ascii 1.0", "comment VCGLIB generated", f"element vertex {W * H}",
             "property float x", "property float y", "property float z", "property uchar red",
             "property uchar green", "property uchar blue", f"element face {(W - 1) * (H - 1)}",
             "property list uchar int vertex_indices", "end_header"]
    v = vertices.reshape(-1, 3)
    c = (f32(colors.reshape(-1, 3) * f32(255.0)).astype(np.int64) if colors is not None
         else np.zeros((W * H, 3), np.int64))
    for i in range(W * H):
        lines.append("%g %g %g %d %d %d " % (float(v[i, 0]), float(v[i, 1]), float(v[i, 2]), c[i, 0], c[i, 1], c[i, 2]))
    for row in range(H - 1):
        for col in range(W - 1):
            a, b = row * W + col, (row + 1) * W + col
            lines.append(f"4 {a} {b} {b + 1} {a + 1} ")
    return "\n".join(lines) + "\n"


def reconstruction(left, right, cams, D, q=None, zscale=1.0, cost="ssd", optimizer="wta", median_filter=True,
                   dilate=True):
    """The reference's reconstruction chain on one pair of 8-bit 3-channel
    frames (tdvision/reconstruction.cpp:9-55): grey conversion and remap of
    both frames and of the left color frame (rectificationcv.cpp:258-310), the
    DevStereoMatcher (5x5 Gaussian, cost, optimizer; devstereomatcher.cpp:13-48,
    commonstereomatcherfactory.cpp:40-80) giving d/D, the opening (dilate.cpp),
    then the reprojection with the rectified left colors.  ``cams`` holds
    (K, dist, R, P) of each camera.  Returns (rectified left color, d/D map,
    vertices, colors)."""
    import oracle as orc
    H, W = left.shape[:2]
    maps = [rectify_maps(K, dist, R, P, W, H) for (K, dist, R, P) in cams]
    gl = remap(to_gray(left), *maps[0])
    gr = remap(to_gray(right), *maps[1])
    cl = remap(left, *maps[0])
    if median_filter:
        gl, gr = gauss5(gl), gauss5(gr)
    C = {"ssd": orc.ssd_cost, "ncc": orc.ncc_cost, "bt": orc.bt_cost}[cost](gl, gr, D)
    if optimizer == "wta":
        _, dn = orc.wta(C)
    elif optimizer == "dp":
        _, dn = orc.dp(C)
    else:
        _, dn, _ = orc.sgm(C, gl, 30.0 / 255.0, 150.0 / 255.0, p2_mode=orc.P2_ADJUST, table=orc.TABLE_REF,
                           semantics=orc.SEM_REF_GPU, want_S=False)
    if dilate:
        dn = open7(dn)
    v, c = reproject(dn, cl, "q" if q is not None else "direct", zscale, q)
    return cl, dn, v, c
