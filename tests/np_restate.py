"""An independent numpy restatement of the reference's CPU path.

Test infrastructure: it cross-checks the C++ oracle (oracle/dsref.cpp). It is
written straight from the Rust sources with whole-array numpy float32
arithmetic in the reference's evaluation order, so on small inputs it must
agree with the oracle bit for bit (NLM up to the last ulp of ``exp``).

  demosaic.rs:90-124   mhc_bayer
  demosaic.rs:147-344  rcd_bayer
  demosaic.rs:31-42    clip_plane
  image.rs:269-313     box_blur
  enhance.rs:36-72     nlm
  demosaic.rs:419-502  cfa_clip_levels, reconstruct_highlights
  image.rs:327-373     gaussian_blur (sigma >= 2), box_radii_for_gauss
"""
from __future__ import annotations

import numpy as np

F = np.float32


def _color_map(pat, h, w):
    pat = np.asarray(pat, np.int64).reshape(2, 2)
    yy, xx = np.mgrid[0:h, 0:w]
    return pat[yy % 2, xx % 2]


def _shift(a, dx, dy, y0, y1, x0, x1):
    """a[y+dy, x+dx] for y in [y0,y1), x in [x0,x1)."""
    return a[y0 + dy:y1 + dy, x0 + dx:x1 + dx]


def mhc(cfa, pat, mul):
    h, w = cfa.shape
    col = _color_map(pat, h, w)
    m = np.asarray(mul, F)[col]
    v_all = (cfa.astype(F) * m).astype(F)
    pad = np.pad(v_all, 2, mode="edge")

    def p(dx, dy):
        return pad[2 + dy:2 + dy + h, 2 + dx:2 + dx + w]

    v = p(0, 0)
    g_at_rb = (F(4) * v + F(2) * (p(0, -1) + p(-1, 0) + p(1, 0) + p(0, 1)) - (p(0, -2) + p(-2, 0) + p(2, 0) + p(0, 2))) / F(8)
    rb_g_row = (F(5) * v + F(4) * (p(-1, 0) + p(1, 0)) - (p(-2, 0) + p(2, 0) + p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1))
                + F(0.5) * (p(0, -2) + p(0, 2))) / F(8)
    rb_g_col = (F(5) * v + F(4) * (p(0, -1) + p(0, 1)) - (p(0, -2) + p(0, 2) + p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1))
                + F(0.5) * (p(-2, 0) + p(2, 0))) / F(8)
    rb_diag = (F(6) * v + F(2) * (p(-1, -1) + p(1, -1) + p(-1, 1) + p(1, 1)) - F(1.5) * (p(0, -2) + p(-2, 0) + p(2, 0) + p(0, 2))) / F(8)
    patarr = np.asarray(pat, np.int64).reshape(2, 2)
    yy, xx = np.mgrid[0:h, 0:w]
    row_c = patarr[yy % 2, (xx + 1) % 2]
    out = np.zeros((h, w, 3), F)
    g_site = col == 1
    r_row = g_site & (row_c == 0)
    b_row = g_site & (row_c != 0)
    out[..., 0] = np.where(col == 0, v, np.where(col == 2, rb_diag, np.where(r_row, rb_g_row, rb_g_col)))
    out[..., 1] = np.where(g_site, v, g_at_rb)
    out[..., 2] = np.where(col == 2, v, np.where(col == 0, rb_diag, np.where(r_row, rb_g_col, rb_g_row)))
    del b_row
    return np.fmax(out, F(0))


def rcd(cfa, pat, mul):
    h, w = cfa.shape
    if w < 16 or h < 16:
        return mhc(cfa, pat, mul)
    col = _color_map(pat, h, w)
    c = np.fmax(cfa.astype(F) * np.asarray(mul, F)[col], F(0))
    eps = F(1e-5)
    S = lambda a, dx, dy, y0, y1, x0, x1: _shift(a, dx, dy, y0, y1, x0, x1)

    # step 1
    bv = np.zeros((h, w), F)
    bh = np.zeros((h, w), F)
    r0 = (3, h - 3, 3, w - 3)
    cc = lambda dx, dy: S(c, dx, dy, *r0)
    t = (cc(0, -3) - cc(0, -1) - cc(0, 1) + cc(0, 3)) - F(3) * (cc(0, -2) + cc(0, 2)) + F(6) * cc(0, 0)
    bv[3:h - 3, 3:w - 3] = t * t
    t = (cc(-3, 0) - cc(-1, 0) - cc(1, 0) + cc(3, 0)) - F(3) * (cc(-2, 0) + cc(2, 0)) + F(6) * cc(0, 0)
    bh[3:h - 3, 3:w - 3] = t * t
    vh = np.full((h, w), F(0.5))
    r4 = (4, h - 4, 4, w - 4)
    vs = np.fmax(S(bv, 0, -1, *r4) + S(bv, 0, 0, *r4) + S(bv, 0, 1, *r4), eps)
    hs = np.fmax(S(bh, -1, 0, *r4) + S(bh, 0, 0, *r4) + S(bh, 1, 0, *r4), eps)
    vh[4:h - 4, 4:w - 4] = vs / (vs + hs)

    # step 2
    lpf = np.zeros((h, w), F)
    r2 = (2, h - 2, 2, w - 2)
    c2 = lambda dx, dy: S(c, dx, dy, *r2)
    v = c2(0, 0) + F(0.5) * (c2(0, -1) + c2(0, 1) + c2(-1, 0) + c2(1, 0)) + F(0.25) * (
        c2(-1, -1) + c2(1, -1) + c2(-1, 1) + c2(1, 1))
    lpf[2:h - 2, 2:w - 2] = np.where(col[2:h - 2, 2:w - 2] == 1, F(0), v)

    base = mhc(cfa, pat, mul)
    r = np.where(col == 0, c, base[..., 0])
    g = np.where(col == 1, c, base[..., 1])
    b = np.where(col == 2, c, base[..., 2])

    def disc(d):
        central = S(d, 0, 0, *r4)
        neigh = F(0.25) * (S(d, -1, -1, *r4) + S(d, 1, -1, *r4) + S(d, -1, 1, *r4) + S(d, 1, 1, *r4))
        return np.where(np.abs(F(0.5) - central) < np.abs(F(0.5) - neigh), neigh, central)

    # step 3
    c4 = lambda dx, dy: S(c, dx, dy, *r4)
    l4 = lambda dx, dy: S(lpf, dx, dy, *r4)
    vd = disc(vh)
    n_grad = eps + np.abs(c4(0, -1) - c4(0, 1)) + np.abs(c4(0, 0) - c4(0, -2)) + np.abs(c4(0, -1) - c4(0, -3)) + np.abs(c4(0, -2) - c4(0, -4))
    s_grad = eps + np.abs(c4(0, -1) - c4(0, 1)) + np.abs(c4(0, 0) - c4(0, 2)) + np.abs(c4(0, 1) - c4(0, 3)) + np.abs(c4(0, 2) - c4(0, 4))
    w_grad = eps + np.abs(c4(-1, 0) - c4(1, 0)) + np.abs(c4(0, 0) - c4(-2, 0)) + np.abs(c4(-1, 0) - c4(-3, 0)) + np.abs(c4(-2, 0) - c4(-4, 0))
    e_grad = eps + np.abs(c4(-1, 0) - c4(1, 0)) + np.abs(c4(0, 0) - c4(2, 0)) + np.abs(c4(1, 0) - c4(3, 0)) + np.abs(c4(2, 0) - c4(4, 0))
    n_est = c4(0, -1) * F(2) * l4(0, 0) / (eps + l4(0, 0) + l4(0, -2))
    s_est = c4(0, 1) * F(2) * l4(0, 0) / (eps + l4(0, 0) + l4(0, 2))
    w_est = c4(-1, 0) * F(2) * l4(0, 0) / (eps + l4(0, 0) + l4(-2, 0))
    e_est = c4(1, 0) * F(2) * l4(0, 0) / (eps + l4(0, 0) + l4(2, 0))
    with np.errstate(invalid="ignore", divide="ignore"):
        v_est = (s_grad * n_est + n_grad * s_est) / (n_grad + s_grad)
        h_est = (w_grad * e_est + e_grad * w_est) / (e_grad + w_grad)
    gnew = np.fmax(vd * h_est + (F(1) - vd) * v_est, F(0))
    inner = col[4:h - 4, 4:w - 4]
    g[4:h - 4, 4:w - 4] = np.where(inner == 1, g[4:h - 4, 4:w - 4], gnew)

    # step 4.1/4.2
    bp = np.zeros((h, w), F)
    bq = np.zeros((h, w), F)
    t = (cc(-3, -3) - cc(-1, -1) - cc(1, 1) + cc(3, 3)) - F(3) * (cc(-2, -2) + cc(2, 2)) + F(6) * cc(0, 0)
    bp[3:h - 3, 3:w - 3] = t * t
    t = (cc(3, -3) - cc(1, -1) - cc(-1, 1) + cc(-3, 3)) - F(3) * (cc(2, -2) + cc(-2, 2)) + F(6) * cc(0, 0)
    bq[3:h - 3, 3:w - 3] = t * t
    pq = np.full((h, w), F(0.5))
    ps = np.fmax(S(bp, -1, -1, *r4) + S(bp, 0, 0, *r4) + S(bp, 1, 1, *r4), eps)
    qs = np.fmax(S(bq, 1, -1, *r4) + S(bq, 0, 0, *r4) + S(bq, -1, 1, *r4), eps)
    pq[4:h - 4, 4:w - 4] = ps / (ps + qs)

    def pass43(target, at_color):
        ch = target.copy()
        k = lambda dx, dy: S(ch, dx, dy, *r4)
        gg = lambda dx, dy: S(g, dx, dy, *r4)
        pd = disc(pq)
        nw_g = eps + np.abs(k(-1, -1) - k(1, 1)) + np.abs(k(-1, -1) - k(-3, -3)) + np.abs(gg(0, 0) - gg(-2, -2))
        ne_g = eps + np.abs(k(1, -1) - k(-1, 1)) + np.abs(k(1, -1) - k(3, -3)) + np.abs(gg(0, 0) - gg(2, -2))
        sw_g = eps + np.abs(k(-1, 1) - k(1, -1)) + np.abs(k(-1, 1) - k(-3, 3)) + np.abs(gg(0, 0) - gg(-2, 2))
        se_g = eps + np.abs(k(1, 1) - k(-1, -1)) + np.abs(k(1, 1) - k(3, 3)) + np.abs(gg(0, 0) - gg(2, 2))
        nw_e = k(-1, -1) - gg(-1, -1)
        ne_e = k(1, -1) - gg(1, -1)
        sw_e = k(-1, 1) - gg(-1, 1)
        se_e = k(1, 1) - gg(1, 1)
        p_est = (nw_g * se_e + se_g * nw_e) / (nw_g + se_g)
        q_est = (ne_g * sw_e + sw_g * ne_e) / (ne_g + sw_g)
        val = np.fmax(gg(0, 0) + (F(1) - pd) * p_est + pd * q_est, F(0))
        target[4:h - 4, 4:w - 4] = np.where(inner == at_color, val, target[4:h - 4, 4:w - 4])

    pass43(r, 2)
    pass43(b, 0)

    def pass44(target):
        ch = target.copy()
        k = lambda dx, dy: S(ch, dx, dy, *r4)
        gg = lambda dx, dy: S(g, dx, dy, *r4)
        vd = disc(vh)
        n_g = eps + np.abs(gg(0, 0) - gg(0, -2)) + np.abs(k(0, -1) - k(0, 1)) + np.abs(k(0, -1) - k(0, -3))
        s_g = eps + np.abs(gg(0, 0) - gg(0, 2)) + np.abs(k(0, 1) - k(0, -1)) + np.abs(k(0, 1) - k(0, 3))
        w_g = eps + np.abs(gg(0, 0) - gg(-2, 0)) + np.abs(k(-1, 0) - k(1, 0)) + np.abs(k(-1, 0) - k(-3, 0))
        e_g = eps + np.abs(gg(0, 0) - gg(2, 0)) + np.abs(k(1, 0) - k(-1, 0)) + np.abs(k(1, 0) - k(3, 0))
        n_e = k(0, -1) - gg(0, -1)
        s_e = k(0, 1) - gg(0, 1)
        w_e = k(-1, 0) - gg(-1, 0)
        e_e = k(1, 0) - gg(1, 0)
        v_est = (n_g * s_e + s_g * n_e) / (n_g + s_g)
        h_est = (e_g * w_e + w_g * e_e) / (e_g + w_g)
        val = np.fmax(gg(0, 0) + (F(1) - vd) * v_est + vd * h_est, F(0))
        target[4:h - 4, 4:w - 4] = np.where(inner == 1, val, target[4:h - 4, 4:w - 4])

    pass44(r)
    pass44(b)
    return np.stack([r, g, b], axis=-1).astype(F)


def clip_plane(cfa):
    raw = (cfa >= F(0.995)).astype(F)
    pad = np.pad(raw, 1, mode="edge")
    h, w = cfa.shape
    m = np.zeros((h, w), F)
    for dy in range(3):
        for dx in range(3):
            m = np.fmax(m, pad[dy:dy + h, dx:dx + w])
    return m


def box_blur(p, r):
    if r == 0 or p.size == 0:
        return p.copy()
    h, w = p.shape
    dt = p.dtype.type
    norm = dt(1) / dt(2 * r + 1)

    def run(a, n):  # running sum along axis 1 of a (rows x n), clamped edges
        acc = np.zeros(a.shape[0], dt)
        for i in range(-r, r + 1):
            acc = acc + a[:, min(max(i, 0), n - 1)]
        xs = np.arange(n - 1)
        hi = np.clip(xs + r + 1, 0, n - 1)
        lo = np.clip(xs - r, 0, n - 1)
        d = a[:, hi] - a[:, lo]
        seq = np.concatenate([acc[:, None], d], axis=1)
        return np.add.accumulate(seq, axis=1, dtype=dt) * norm

    tmp = run(p, w)
    out = run(tmp.T.copy(), h).T
    return np.ascontiguousarray(out)


def nlm(p, h_param, search, patch, nthreads=1):
    dt = p.dtype.type
    h, w = p.shape
    h2 = max(dt(h_param) * dt(h_param), dt(1e-12))
    offs = [(dx, dy) for dy in range(-search, search + 1) for dx in range(-search, search + 1)]
    pad = np.pad(p, max(search, 0), mode="edge")
    csz = max(-(-len(offs) // max(nthreads, 1)), 1)
    chunks = [offs[i:i + csz] for i in range(0, len(offs), csz)]
    acc = np.zeros_like(p)
    wsum = np.zeros_like(p)
    for ch in chunks:
        a = np.zeros_like(p)
        s = np.zeros_like(p)
        for dx, dy in ch:
            q = pad[search + dy:search + dy + h, search + dx:search + dx + w]
            d = p - q
            dist = box_blur(d * d, patch)
            x = -(dist / h2)
            wt = np.exp(x.astype(np.float64)).astype(dt) if dt is np.float32 else np.exp(x)
            a = a + wt * q
            s = s + wt
        acc = acc + a
        wsum = wsum + s
    return acc / np.fmax(wsum, dt(1e-12))


FMAX = F(np.finfo(F).max)


def cfa_clip_levels(cfa, pat):
    h, w = cfa.shape
    cm = _color_map(pat, h, w)[::3]
    rows = cfa[::3]
    mx = np.zeros(3, F)
    for c in range(3):
        v = rows[cm == c]
        if v.size:
            mx[c] = np.fmax(F(0), v.max())
    return np.where(mx >= F(0.95), mx, FMAX).astype(F)


def _round_half_away(x):
    return int(np.sign(x) * np.floor(abs(float(x)) + 0.5))


def box_radii_for_gauss(sigma, n=3):
    sigma, nf = F(sigma), F(n)
    w_ideal = np.sqrt(F(12) * sigma * sigma / nf + F(1))
    wl = int(np.floor(w_ideal))
    if wl % 2 == 0:
        wl -= 1
    wu = wl + 2
    m_ideal = (F(12) * sigma * sigma - F(n * wl * wl) - F(4) * nf * F(wl) - F(3) * nf) / (F(-4) * F(wl) - F(4))
    m = _round_half_away(m_ideal)
    return [max(((wl if i < m else wu) - 1) // 2, 0) for i in range(n)]


def gaussian_blur(p, sigma):
    r = box_radii_for_gauss(sigma, 3)
    return box_blur(box_blur(box_blur(p, r[0]), r[1]), r[2])


def reconstruct_highlights(img, clip, mul, raw_clip):
    img = np.asarray(img, F)
    if not (clip > 0).any():
        return img.copy()
    lvl = [FMAX if F(raw_clip[c]) == FMAX else F(raw_clip[c]) * F(mul[c]) * F(0.97) for c in range(3)]
    P = [img[..., c] for c in range(3)]
    cl = [(P[c] >= lvl[c]) | ((clip > 0) & (P[c] >= lvl[c] * F(0.8))) for c in range(3)]
    h, w = clip.shape
    sigma = max(F(max(w, h)) / F(120), F(2))
    lmin = min(min(min(lvl[0], lvl[1]), lvl[2]), F(4))
    near = box_blur(clip.astype(F), 3)
    valid = ~((near > 0) | cl[0] | cl[1] | cl[2] | (P[1] <= F(1e-4)))
    with np.errstate(all="ignore"):
        y = (P[0] + P[1] + P[2]) / F(3) / lmin
        k = np.minimum(y * y, F(1))
        rr = np.clip(P[0] / P[1], F(0.1), F(10)) * k
        br = np.clip(P[2] / P[1], F(0.1), F(10)) * k
    z = F(0)
    wgt, rr, br = (np.where(valid, a, z).astype(F) for a in (k, rr, br))
    wb, rrb, brb = (gaussian_blur(a, sigma) for a in (wgt, rr, br))
    nc = cl[0].astype(np.int32) + cl[1] + cl[2]
    m = np.fmax(np.fmax(P[0], P[1]), P[2])
    with np.errstate(all="ignore"):
        big = wb > F(1e-4)
        r = np.where(big, rrb / wb, F(1)).astype(F)
        b = np.where(big, brb / wb, F(1)).astype(F)
    trust = np.minimum(wb * F(3), F(1))
    r = F(1) + (r - F(1)) * trust
    b = F(1) + (b - F(1)) * trust
    ratio = [r, np.ones_like(r), b]
    g = P[1].copy()
    with np.errstate(all="ignore"):
        for c in range(3):
            g = np.where(~cl[c], np.fmax(g, P[c] / ratio[c]), g)
    q = [np.where(cl[c], np.fmax(P[c], g * ratio[c]), P[c]) for c in range(3)]
    top = np.fmax(np.fmax(q[0], q[1]), q[2])
    t = (nc.astype(F) / F(3)) * (nc.astype(F) / F(3))
    q = [q[c] + (top - q[c]) * t * F(0.5) for c in range(3)]
    out = np.stack(q, axis=-1)
    out = np.where((nc == 3)[..., None], m[..., None], out)
    out = np.where((nc == 0)[..., None], img, out)
    return out.astype(F)
