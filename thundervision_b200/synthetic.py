"""Seeded synthetic rectified stereo pairs (stand-in for the reference's image
pairs: Tsukuba / Teddy / Cones under res/, swept by
BenchmarkApp/src/run_tests.py:10-22).

Every pair is grey uint8.  The left image is uniform noise blurred with a
Gaussian and rescaled to 0..255; the right image is the left image forward-
warped by an integer disparity field (x_r = x - d), nearer surfaces (larger d)
winning, disoccluded right pixels filled with fresh noise; then additive
Gaussian sensor noise and clipping.  Ground truth is the left disparity field.

Recipes:
  pair_small   384x288, D=16: background d=2, 4 rectangles d in [0,15].
  pair_medium  640x480, D=64: background d=2, one slanted-plane rectangle
               (d linear in x from 10 to 50), 8 rectangles d in [0,63],
               then 2 % salt-and-pepper on both images.
  video_frames 1920x1080, D=256: slanted background (d 8..64 linear in x),
               12 rectangles (d in [24,200]) moving at integer 1..4 px/frame.
"""
import numpy as np

_SEED_MIX = 0x9E3779B97F4A7C15


def pair_seed(seed, index):
    """Per-pair seed = hash(seed, index) (splitmix64 finaliser)."""
    z = (int(seed) * _SEED_MIX + int(index) + 1) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return z ^ (z >> 31)


def _gauss_kernel(sigma):
    r = max(1, int(np.ceil(3 * sigma)))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    return k / k.sum()


def _blur(img, sigma):
    k = _gauss_kernel(sigma)
    r = len(k) // 2
    p = np.pad(img, ((0, 0), (r, r)), mode="reflect")
    tmp = np.zeros_like(img)
    for i, w in enumerate(k):
        tmp += w * p[:, i:i + img.shape[1]]
    p = np.pad(tmp, ((r, r), (0, 0)), mode="reflect")
    out = np.zeros_like(img)
    for i, w in enumerate(k):
        out += w * p[i:i + img.shape[0], :]
    return out


def _texture(rng, H, W, sigma=1.5):
    n = rng.uniform(0.0, 255.0, size=(H, W))
    b = _blur(n, sigma)
    lo, hi = b.min(), b.max()
    return np.round((b - lo) * (255.0 / max(hi - lo, 1e-9)))


def _warp(left, disp, rng, noise_sigma=2.0):
    """Forward-warp left by disp (x_r = x - d); larger d wins; holes get fresh
    noise; add N(0, sigma^2) and clip to uint8."""
    H, W = left.shape
    right = np.full((H, W), np.nan)
    zbuf = np.full((H, W), -1, np.int64)
    ys, xs = np.mgrid[0:H, 0:W]
    xr = xs - disp
    ok = xr >= 0
    order = np.argsort(disp[ok], kind="stable")
    yy, xx, rr, dd = ys[ok][order], xs[ok][order], xr[ok][order], disp[ok][order]
    # ascending d: later (nearer) writes overwrite
    right[yy, rr] = left[yy, xx]
    zbuf[yy, rr] = dd
    holes = np.isnan(right)
    right[holes] = rng.uniform(0.0, 255.0, size=int(holes.sum()))
    occl = np.ones((H, W), bool)
    visible = zbuf[ys[ok], xr[ok]] == disp[ok]
    occl[ys[ok][visible], xs[ok][visible]] = False
    right = right + rng.normal(0.0, noise_sigma, size=(H, W))
    return np.clip(np.round(right), 0, 255).astype(np.uint8), occl


def _rects(rng, H, W, n, dlo, dhi):
    out = []
    for _ in range(n):
        rw = int(rng.integers(max(4, W // 12), max(5, W // 4)))
        rh = int(rng.integers(max(4, H // 12), max(5, H // 4)))
        x0 = int(rng.integers(0, max(1, W - rw)))
        y0 = int(rng.integers(0, max(1, H - rh)))
        d = int(rng.integers(dlo, dhi + 1))
        out.append((x0, y0, rw, rh, d))
    return out


def _salt_pepper(img, rng, frac):
    m = rng.random(img.shape) < frac
    vals = np.where(rng.random(img.shape) < 0.5, 0, 255).astype(np.uint8)
    out = img.copy()
    out[m] = vals[m]
    return out


def make_pair(W, H, D, seed, n_rects=4, slanted=False, salt_pepper=0.0, background=2):
    rng = np.random.default_rng(seed)
    left = _texture(rng, H, W)
    disp = np.full((H, W), min(background, D - 1), np.int64)
    if slanted:
        sw, sh = W // 2, H // 2
        sx0 = int(rng.integers(0, W - sw))
        sy0 = int(rng.integers(0, H - sh))
        ramp = np.round(10 + 40 * np.arange(sw) / max(sw - 1, 1)).astype(np.int64)
        disp[sy0:sy0 + sh, sx0:sx0 + sw] = np.minimum(ramp[None, :], D - 1)
    for (x0, y0, rw, rh, d) in _rects(rng, H, W, n_rects, 0, D - 1):
        disp[y0:y0 + rh, x0:x0 + rw] = d
    right, occl = _warp(left, disp, rng)
    left = np.clip(np.round(left + rng.normal(0.0, 2.0, size=(H, W))), 0, 255).astype(np.uint8)
    if salt_pepper > 0:
        left = _salt_pepper(left, rng, salt_pepper)
        right = _salt_pepper(right, rng, salt_pepper)
    return left, right, disp.astype(np.uint16), occl


def pair_small(seed=0):
    """384x288, D=16, 4 rectangles over background 2."""
    return make_pair(384, 288, 16, seed, n_rects=4)


def pair_medium(seed=0):
    """640x480, D=64, 8 rectangles + slanted plane, 2 % salt-and-pepper."""
    return make_pair(640, 480, 64, seed, n_rects=8, slanted=True, salt_pepper=0.02)


def pair_sized(W, H, D, seed):
    """Generic pair generated like pair_medium at any size."""
    return make_pair(W, H, D, seed, n_rects=8, slanted=True, salt_pepper=0.02)


class VideoStream:
    """1920x1080 (by default) frames: slanted background plus moving rectangles."""

    def __init__(self, W=1920, H=1080, D=256, seed=0, n_rects=12):
        self.W, self.H, self.D = W, H, D
        self.rng = np.random.default_rng(seed)
        self.left_tex = _texture(self.rng, H, W + 512)
        self.rects = []
        for (x0, y0, rw, rh, d) in _rects(self.rng, H, W, n_rects, min(24, D - 1), min(200, D - 1)):
            vx = int(self.rng.integers(1, 5)) * (1 if self.rng.random() < 0.5 else -1)
            vy = int(self.rng.integers(1, 5)) * (1 if self.rng.random() < 0.5 else -1)
            self.rects.append([x0, y0, rw, rh, d, vx, vy])
        self.bg = np.minimum(np.round(8 + 56 * np.arange(W) / (W - 1)).astype(np.int64), D - 1)

    def frame(self, t):
        W, H = self.W, self.H
        rng = np.random.default_rng(pair_seed(12345, t))
        left = self.left_tex[:, (t * 2) % 512:(t * 2) % 512 + W].copy()
        disp = np.broadcast_to(self.bg[None, :], (H, W)).copy()
        for (x0, y0, rw, rh, d, vx, vy) in self.rects:
            x = (x0 + vx * t) % max(1, W - rw)
            y = (y0 + vy * t) % max(1, H - rh)
            disp[y:y + rh, x:x + rw] = d
        right, occl = _warp(left, disp, rng)
        left = np.clip(np.round(left + rng.normal(0.0, 2.0, size=(H, W))), 0, 255).astype(np.uint8)
        return left, right, disp.astype(np.uint16), occl


def batch_shapes(seed=0, n=64):
    """Config of the uneven batch: W ~ U[320,1920], H ~ U[240,1080] rounded to
    multiples of 16, D in {32,64,128,256}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        W = int(round(rng.uniform(320, 1920) / 16)) * 16
        H = int(round(rng.uniform(240, 1080) / 16)) * 16
        D = int(rng.choice([32, 64, 128, 256]))
        out.append((W, H, D))
    return out
