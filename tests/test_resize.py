"""Working-resolution images (load_views, mvs/src/lib.rs:183-194): the
`image` 0.24 Triangle resize_exact followed by to_luma8 / to_rgb8.  The
oracle is checked against hand-derived answers and an independent numpy
restatement; the GPU path (rcmvs_resize_view) against the oracle, bit for
bit."""
import numpy as np
import pytest

from oracle import oracle
from rustcolmap_b200 import colmap, mvs

F = np.float32


def taps_np(n, m, o):
    """Second restatement of one output sample's taps (numpy f32 scalars)."""
    ratio = F(n) / F(m)
    s = ratio if ratio >= F(1) else F(1)
    c = (F(o) + F(0.5)) * ratio
    left = min(max(int(np.floor(c - s)), 0), n - 1)
    right = min(max(int(np.ceil(c + s)), left + 1), n)
    c = c - F(0.5)
    ws, total = [], F(0)
    for i in range(left, right):
        x = (F(i) - c) / s
        w = F(1) - abs(x) if abs(x) < F(1) else F(0)
        ws.append(F(w))
        total = F(total + w)
    return left, [F(w / total) for w in ws]


def round_half_away(t):
    f = np.floor(t)
    return (f + (t - f >= F(0.5))).astype(np.uint8)


def resize_np(img, mw, mh):
    a = np.asarray(img, np.uint8)
    if a.ndim == 2:
        a = a[:, :, None]
    h, w, ch = a.shape
    nc = 1 if ch < 3 else 3
    a = a[:, :, :nc]
    if (mw, mh) == (w, h):
        px = a
    else:
        tmp = np.empty((mh, w, nc), F)
        for oy in range(mh):
            top, ws = taps_np(h, mh, oy)
            t = np.zeros((w, nc), F)
            for i, wt in enumerate(ws):
                t = t + a[top + i].astype(F) * wt
            tmp[oy] = t
        px = np.empty((mh, mw, nc), np.uint8)
        for ox in range(mw):
            first, ws = taps_np(w, mw, ox)
            t = np.zeros((mh, nc), F)
            for i, wt in enumerate(ws):
                t = t + tmp[:, first + i] * wt
            px[:, ox] = round_half_away(np.clip(t, F(0), F(255)))
    if nc == 1:
        return px[:, :, 0].copy(), np.repeat(px, 3, axis=2)
    p = px.astype(np.uint32)
    g = ((2126 * p[:, :, 0] + 7152 * p[:, :, 1] + 722 * p[:, :, 2]) // 10000).astype(np.uint8)
    return g, px.copy()


def image(seed, h, w, c):
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 256, (h, w, c), dtype=np.uint8)
    # smooth areas and hard edges: gradients plus the noise
    yy, xx = np.mgrid[0:h, 0:w]
    grad = ((xx * 7 + yy * 3) % 256).astype(np.uint8)[:, :, None]
    return np.where(rng.uniform(size=(h, w, 1)) < 0.5, base, grad).astype(np.uint8)


# (h, w, channels, mw, mh): downscales by integer and odd ratios, one axis
# only, upscales, a single row / column, the 16-pixel floor, every channel count
CASES = [
    (64, 96, 1, 48, 32), (64, 96, 3, 70, 47), (61, 97, 3, 23, 17), (40, 40, 1, 40, 17),
    (40, 40, 3, 13, 40), (20, 30, 1, 45, 31), (1, 9, 1, 4, 1), (9, 1, 3, 1, 4), (1, 1, 3, 16, 16),
    (300, 400, 3, 16, 16), (77, 50, 2, 33, 51), (50, 77, 4, 51, 33), (33, 65, 3, 65, 33),
]


# ------------------------------------------------------------------ CPU
def test_oracle_known_answers():
    g, rgb = oracle.resize_view(np.array([[10, 20, 30, 40]], np.uint8), 2, 1)
    # taps of output 0: inputs 0-2 weighted 3:3:1 / 7; of output 1: inputs 1-3, 1:3:3 / 7
    assert g.tolist() == [[17, 33]] and rgb[0, 1].tolist() == [33, 33, 33]
    for h, w, c, mw, mh in CASES:
        img = np.full((h, w, c), 200, np.uint8)
        g, rgb = oracle.resize_view(img, mw, mh)
        # weights sum to 1 within f32 rounding; (2126 + 7152 + 722) / 10000 = 1
        assert (g == 200).all() and (rgb == 200).all(), (h, w, c, mw, mh)
    # no size change: to_luma8 / to_rgb8 only
    img = image(1, 10, 12, 3)
    g, rgb = oracle.resize_view(img, 12, 10)
    g2, rgb2 = colmap.gray_rgb(img)
    assert np.array_equal(g, g2) and np.array_equal(rgb, rgb2)


def test_oracle_matches_numpy_restatement():
    for k, (h, w, c, mw, mh) in enumerate(CASES):
        img = image(k, h, w, c)
        a = oracle.resize_view(img, mw, mh)
        b = resize_np(img, mw, mh)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (h, w, c, mw, mh)


def test_alpha_is_dropped():
    img = image(4, 30, 20, 4)
    other = img.copy()
    other[:, :, 3] = 255 - other[:, :, 3]
    for size in ((20, 30), (11, 7)):
        a, b = oracle.resize_view(img, *size), oracle.resize_view(other, *size)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        c = oracle.resize_view(img[:, :, :3], *size)
        assert np.array_equal(a[0], c[0]) and np.array_equal(a[1], c[1])


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def ctx():
    c = mvs.Context(0)
    yield c
    c.close()


@pytest.mark.gpu
def test_gpu_resize_matches_oracle(ctx):
    for k, (h, w, c, mw, mh) in enumerate(CASES):
        img = image(k, h, w, c)
        g, rgb = mvs.resize_view(img, mw, mh, ctx)
        og, orgb = oracle.resize_view(img, mw, mh)
        assert np.array_equal(g, og) and np.array_equal(rgb, orgb), (h, w, c, mw, mh)


@pytest.mark.gpu
@pytest.mark.parametrize("h,w,c,max_dim", [(3000, 4000, 3, 1920), (3000, 4000, 3, 900), (1080, 1920, 1, 1000),
                                           (2000, 3, 1, 1000)])
def test_gpu_resize_full_size(ctx, h, w, c, max_dim):
    img = image(7, h, w, c)
    mw, mh = mvs.working_size(w, h, max_dim)
    g, rgb = mvs.resize_view(img, mw, mh, ctx)
    og, orgb = oracle.resize_view(img, mw, mh)
    assert np.array_equal(g, og) and np.array_equal(rgb, orgb)
    g2, _ = mvs.resize_view(img, mw, mh, ctx)  # scratch reuse
    assert np.array_equal(g2, g)


@pytest.mark.gpu
def test_gpu_resize_arguments(ctx):
    img = np.zeros((4, 4, 3), np.uint8)
    for mw, mh in ((0, 4), (4, -1), ((1 << 23) + 1, 1)):
        with pytest.raises(mvs.RcmvsError):
            mvs.resize_view(img, mw, mh, ctx)
    with pytest.raises(mvs.RcmvsError):
        mvs.resize_view(np.zeros((4, 4, 5), np.uint8), 2, 2, ctx)


def test_oracle_matches_numpy_random_sizes():
    """Seeded random shapes, ratios (down and up, per axis) and channel counts."""
    rng = np.random.default_rng(2024)
    for k in range(24):
        h, w = (int(v) for v in rng.integers(1, 90, 2))
        c = int(rng.integers(1, 5))
        mh, mw = (int(v) for v in rng.integers(1, 120, 2))
        img = image(100 + k, h, w, c)
        a = oracle.resize_view(img, mw, mh)
        b = resize_np(img, mw, mh)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (h, w, c, mw, mh)
