"""SIFT extraction (sfm-lite/src/sift.rs): the CPU oracle against properties
the reference's algorithm guarantees, and the GPU (rcmvs_extract_sift)
against the oracle.

Parity bar.  The pyramid, the DoGs and the extrema with their fitted
positions and responses use only f32/f64 arithmetic, so the count of
extrema must be equal and every keypoint position exact.  Orientations and
descriptors go through exp / atan2 / sin / cos, whose device and host-libm
results may differ in the last bit; descriptors must agree to 1e-4 per
component, and at most 1% of keypoints may differ (a histogram bin or a
peak decision that sits on an exact boundary)."""
import numpy as np
import pytest

from oracle import oracle
from rustcolmap_b200 import mvs, scene, sift

DESC_TOL = 1e-4


def sift_size(w, h, max_dim):
    """sift.rs:436-444: long side to max_dim when larger, sides >= 1."""
    m = max(w, h)
    if m <= max_dim:
        return w, h
    s = max_dim / m
    r = lambda v: int(np.floor(v * s + 0.5))
    return max(r(w), 1), max(r(h), 1)


def oracle_sift(img, max_dim=1600, max_features=2048, thr=0.0067):
    a = img if img.ndim == 3 else img[:, :, None]
    h, w = a.shape[:2]
    mw, mh = sift_size(w, h, max_dim)
    g, rgb = oracle.resize_view(a, mw, mh)
    return oracle.extract_sift(g, rgb, max_features, thr), (mw, mh)


def blob(h=96, w=128, cx=60.5, cy=40.0, s=5.0):
    yy, xx = np.mgrid[0:h, 0:w]
    v = 30 + 200 * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    return v.astype(np.uint8)


def views():
    sc = scene.corner_room(seed=0)
    big = scene.orbit_room(seed=3, n_views=2, sizes=((960, 720),), n_boxes=20, per_view_sparse=10)
    return [sc.views[0], sc.views[5], big.views[0]]


# ------------------------------------------------------------------ CPU
def test_oracle_flat_image_has_no_features():
    img = np.full((80, 120), 128, np.uint8)
    (pts, desc, col, nraw), _ = oracle_sift(img)
    assert nraw == 0 and len(pts) == 0


def test_oracle_blob():
    """A bright Gaussian blob: keypoints near its centre, unit descriptors
    clipped at 0.2 before the second normalisation."""
    img = blob()
    (pts, desc, col, nraw), _ = oracle_sift(img)
    assert len(pts) > 0 and nraw > 0
    d = np.hypot(pts[:, 0] - 60.5, pts[:, 1] - 40.0)
    assert d.min() < 2.0
    assert np.allclose(np.linalg.norm(desc, axis=1), 1.0, atol=1e-5)
    assert (desc >= 0).all()


def test_oracle_properties_on_rendered_views():
    for v in views()[:2]:
        img = np.ascontiguousarray(v.rgb)
        (pts, desc, col, nraw), (w, h) = oracle_sift(img)
        assert 0 < len(pts) <= 2048 and nraw >= len(set(map(tuple, pts)))
        assert (pts[:, 0] >= 0).all() and (pts[:, 0] <= w - 1).all() and (pts[:, 1] <= h - 1).all()
        # colours: the image at the rounded position (half away from zero)
        px = np.minimum(np.floor(pts + 0.5).astype(int), [w - 1, h - 1])
        assert np.array_equal(col, img[px[:, 1], px[:, 0]])
        assert np.allclose(np.linalg.norm(desc, axis=1), 1.0, atol=1e-5)
        # the cap keeps a prefix of the response-sorted list
        (p10, d10, c10, _), _ = oracle_sift(img, max_features=10)
        assert np.array_equal(p10, pts[:10]) and np.array_equal(d10, desc[:10])


def test_oracle_contrast_threshold_monotone():
    img = np.ascontiguousarray(views()[0].gray)
    n = [oracle_sift(img, thr=t)[0][3] for t in (0.02, 0.0067, 0.003)]
    assert n[0] <= n[1] <= n[2]


# ------------------------------------------------------------------ GPU
def match(g, o):
    """Fraction of GPU keypoints with an oracle keypoint at the exact same
    position whose descriptor agrees within DESC_TOL."""
    gp, gd = g
    op, od = o
    index = {}
    for i, p in enumerate(map(tuple, op)):
        index.setdefault(p, []).append(i)
    ok = 0
    for i, p in enumerate(map(tuple, gp)):
        cands = index.get(p, [])
        if cands and min(np.abs(od[j] - gd[i]).max() for j in cands) <= DESC_TOL:
            ok += 1
    return ok / max(len(gp), 1)


@pytest.fixture(scope="module")
def ctx():
    from rustcolmap_b200 import mvs
    c = mvs.Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("k,channels,max_dim,cap", [(0, 3, 1600, 2048), (1, 1, 1600, 2048), (2, 3, 1600, 2048),
                                                    (2, 1, 700, 2048), (0, 4, 200, 2048), (2, 3, 1600, 100000),
                                                    (1, 3, 1600, 7)])
def test_gpu_sift_matches_oracle(ctx, k, channels, max_dim, cap):
    v = views()[k]
    img = np.ascontiguousarray(v.gray if channels == 1 else v.rgb)
    if channels == 4:
        img = np.concatenate([img, np.full(img.shape[:2] + (1,), 77, np.uint8)], axis=2)
    opts = sift.SiftOptions(max_dim=max_dim, max_features=cap)
    f = sift.extract_sift(img, "v", opts, ctx)
    (pts, desc, col, nraw), (w, h) = oracle_sift(img, max_dim, max_features=cap)
    assert np.array_equal(f.colors, col) or len(f.pts) != len(pts)
    assert (f.width, f.height) == (w, h)
    assert f.n_raw == nraw, "scale-space extrema differ"
    assert abs(len(f.pts) - len(pts)) <= max(1, len(pts) // 100)
    assert match((f.pts, f.desc), (pts, desc)) >= 0.99
    same = min(len(pts), len(f.pts))
    exact = np.mean([np.array_equal(f.pts[i], pts[i]) for i in range(same)])
    print(f"\n{w}x{h} c={channels}: {len(f.pts)} keypoints, {nraw} extrema, "
          f"{exact:.4f} in identical order, max desc diff "
          f"{np.abs(f.desc[:same] - desc[:same]).max() if same else 0:.2e}")
    assert np.allclose(np.linalg.norm(f.desc, axis=1), 1.0, atol=1e-5)


@pytest.mark.gpu
def test_gpu_sift_edge_cases(ctx):
    f = sift.extract_sift(np.full((50, 70), 9, np.uint8), ctx=ctx)
    assert len(f.pts) == 0 and f.n_raw == 0
    f = sift.extract_sift(np.zeros((1, 1), np.uint8), ctx=ctx)
    assert len(f.pts) == 0 and (f.width, f.height) == (1, 1)
    img = blob()
    f = sift.extract_sift(img, ctx=ctx)
    (pts, desc, _, nraw), _ = oracle_sift(img)
    assert f.n_raw == nraw and match((f.pts, f.desc), (pts, desc)) >= 0.99
    f10 = sift.extract_sift(np.ascontiguousarray(views()[0].rgb), opts=sift.SiftOptions(max_features=10), ctx=ctx)
    assert len(f10.pts) == 10
    with pytest.raises(sift.RcmvsError):
        sift.extract_sift(np.zeros((4, 4, 5), np.uint8), ctx=ctx)


# ------------------------------------------------------------------ matching
def match_numpy(a, b, ratio=0.8):
    """Second restatement of match_pair: the same serial f32 sums,
    vectorised over the pairs of descriptors."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    if len(a) == 0 or len(b) == 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    s = np.zeros((len(a), len(b)), np.float32)
    for k in range(128):
        d = a[:, None, k] - b[None, :, k]
        s = s + d * d

    def two(m):  # first minimum and second smallest, row-wise
        idx = np.argmin(m, axis=1)
        best = m[np.arange(len(m)), idx]
        rest = m.copy()
        rest[np.arange(len(m)), idx] = np.inf
        return idx, best, rest.min(axis=1)
    fi, f1, f2 = two(s)
    bi, b1, b2 = two(s.T)
    r = np.float32(ratio)
    oa, ob = [], []
    for i in range(len(a)):
        if not np.isfinite(f2[i]) or f1[i] > np.float32(0.9) or f1[i] > r * f2[i]:
            continue
        j = fi[i]
        if bi[j] != i or not np.isfinite(b2[j]) or b1[j] > r * b2[j]:
            continue
        oa.append(i)
        ob.append(j)
    return np.array(oa, np.uint32), np.array(ob, np.uint32)


def desc_sets(seed, na, nb, noise=0.02, dup=0):
    rng = np.random.default_rng(seed)
    a = rng.random((na, 128)).astype(np.float32)
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    perm = rng.permutation(max(na, nb))[:nb] % max(na, 1)
    b = (a[perm] if na else rng.random((nb, 128)).astype(np.float32)) + rng.normal(0, noise, (nb, 128)).astype(np.float32)
    b = np.abs(b)
    b /= np.maximum(np.linalg.norm(b, axis=1, keepdims=True), 1e-12)
    if dup and nb > dup:
        b[-dup:] = b[:dup]  # exact duplicates: equal distances, index ties
    return a, b.astype(np.float32)


def test_oracle_match_pair_known_answers():
    a, _ = desc_sets(0, 50, 50)
    ma, mb = oracle.match_pair(a, a)
    assert np.array_equal(ma, np.arange(50)) and np.array_equal(mb, np.arange(50))
    ma, mb = oracle.match_pair(a, a[::-1])
    assert np.array_equal(mb, 49 - ma) and len(ma) == 50
    # a noisy copy with its first five rows twice: those five are ambiguous
    # (equal nonzero best and second distances fail the ratio test) ...
    noisy = a + np.float32(0.01) * desc_sets(9, 50, 50)[0]
    dup = np.concatenate([noisy, noisy[:5]])
    ma, mb = oracle.match_pair(a, dup)
    assert ma.tolist() == list(range(5, 50)) and mb.tolist() == list(range(5, 50))
    # ... while an exact duplicate at distance 0 passes (0 > 0.8 * 0 is false)
    ma, mb = oracle.match_pair(a, np.concatenate([a, a[:5]]))
    assert ma.tolist() == list(range(50))
    assert len(oracle.match_pair(a[:0], a)[0]) == 0 and len(oracle.match_pair(a, a[:1])[0]) == 0


@pytest.mark.parametrize("na,nb,noise,dup", [(120, 90, 0.02, 0), (64, 64, 0.05, 7), (1, 40, 0.0, 0), (33, 2, 0.01, 0)])
def test_oracle_match_pair_matches_numpy(na, nb, noise, dup):
    a, b = desc_sets(na * nb, na, nb, noise, dup)
    for ratio in (0.8, 0.6):
        x = oracle.match_pair(a, b, ratio)
        y = match_numpy(a, b, ratio)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])


@pytest.mark.gpu
def test_gpu_match_pairs_matches_oracle(ctx):
    sets = [desc_sets(1, 300, 250, 0.03, 6)[0], desc_sets(1, 300, 250, 0.03, 6)[1], desc_sets(2, 65, 129)[1],
            desc_sets(3, 1, 1)[0], np.zeros((0, 128), np.float32)]
    v = views()
    f0 = sift.extract_sift(np.ascontiguousarray(v[0].rgb), ctx=ctx)
    f1 = sift.extract_sift(np.ascontiguousarray(v[1].rgb), ctx=ctx)
    sets += [f0.desc, f1.desc]
    pairs = [(0, 1), (1, 0), (0, 2), (2, 1), (3, 0), (0, 3), (4, 0), (1, 4), (5, 6), (6, 5), (5, 5), (2, 2)]
    for ratio in (0.8, 0.7):
        got = sift.match_pairs(sets, pairs, ratio, ctx)
        for (i, j), (ga, gb) in zip(pairs, got):
            oa, ob = oracle.match_pair(sets[i], sets[j], ratio)
            assert np.array_equal(ga, oa) and np.array_equal(gb, ob), (i, j, ratio)
    ga, gb = sift.match_pair(f0, f1, ctx=ctx)
    assert len(ga) > 50
    print(f"\nSIFT 384x288 views 0 and 5: {len(ga)} mutual matches of {len(f0.pts)} x {len(f1.pts)}")


def test_job_pairs():
    assert sift.job_pairs(4) == [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    assert sift.job_pairs(5, sequential=True) == [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (1, 4), (2, 3), (2, 4),
                                                  (3, 4)]
    assert sift.job_pairs(1) == [] and sift.job_pairs(2, True) == [(0, 1)]
    with pytest.raises(sift.RcmvsError):
        sift.extract_and_match([np.zeros((8, 8), np.uint8)])


@pytest.mark.gpu
def test_extract_and_match_pipeline(ctx):
    sc = scene.corner_room(seed=4, n_views=4, w=160, h=120, f=180.0, arc_deg=30.0, n_patches=40, per_view_sparse=10)
    imgs = [np.ascontiguousarray(v.rgb) for v in sc.views]
    frames, pairs, matches = sift.extract_and_match(imgs, sequential=True, ctx=ctx)
    assert pairs == sift.job_pairs(4, True) and len(matches) == len(pairs)
    for (i, j), (a, b) in zip(pairs, matches):
        oa, ob = oracle.match_pair(frames[i].desc, frames[j].desc, 0.75)
        assert np.array_equal(a, oa) and np.array_equal(b, ob)
    assert sum(len(a) for a, _ in matches) > 0


@pytest.mark.gpu
def test_extract_sift_many_equals_one_context(ctx):
    """Spreading the images over three contexts (streams + host threads)
    gives every image's single-context frame bit for bit, in image order."""
    sc = scene.corner_room(seed=6, n_views=7, w=200, h=150, f=220.0, arc_deg=40.0, n_patches=40, per_view_sparse=10)
    imgs = [np.ascontiguousarray(v.rgb) for v in sc.views] + [np.ascontiguousarray(sc.views[0].gray)]
    one = [sift.extract_sift(im, ctx=ctx) for im in imgs]
    extra = [mvs.Context(0), mvs.Context(0)]
    try:
        many = sift.extract_sift_many(imgs, ctxs=[ctx] + extra)
    finally:
        for c in extra:
            c.close()
    assert len(many) == len(one)
    for a, b in zip(one, many):
        assert (a.width, a.height, a.n_raw) == (b.width, b.height, b.n_raw)
        for x, y in ((a.pts, b.pts), (a.desc, b.desc), (a.colors, b.colors)):
            assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8))


def test_oracle_match_pair_matches_numpy_random():
    """Seeded random set sizes, noise, duplicate counts and ratios."""
    rng = np.random.default_rng(77)
    for k in range(12):
        na, nb = (int(v) for v in rng.integers(1, 90, 2))
        noise = float(rng.choice([0.0, 0.005, 0.03, 0.1]))
        dup = int(rng.integers(0, 4))
        a, b = desc_sets(1000 + k, na, nb, noise, dup)
        ratio = float(rng.choice([0.6, 0.75, 0.8, 0.95]))
        x = oracle.match_pair(a, b, ratio)
        y = match_numpy(a, b, ratio)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), (na, nb, noise, dup, ratio)


def test_image_files(tmp_path):
    for n in ("b.JPG", "a.png", "c.txt", "d.webp", "e.tiff", "noext"):
        (tmp_path / n).write_bytes(b"x")
    (tmp_path / "dir.png").mkdir()
    got = [p.rsplit("/", 1)[1] for p in sift.image_files(str(tmp_path))]
    assert got == ["a.png", "b.JPG", "d.webp", "e.tiff"]
