"""FP64 CPU restatement of the tile feature extractor (features.cu) and of
the diagonal-sweep tile layout, for checking the device features."""
import numpy as np

LB_LAGS, LB_ROWS = 896, 4032


def stats(x, m):
    """Window mean and 1/std (two-pass, population; 0 for flat windows)."""
    s = x.size - m + 1
    W = np.lib.stride_tricks.sliding_window_view(x, m)[:s]
    mu = W.mean(1)
    sd = np.sqrt(((W - mu[:, None]) ** 2).sum(1) / m)
    rms = np.sqrt(mu * mu + sd * sd)
    flat = ~(sd > 1e-12 * rms) | (sd == 0.0)
    isg = np.where(flat, 0.0, 1.0 / np.where(flat, 1.0, sd))
    return mu, isg


def envelope(x, w):
    n = x.size
    U = np.empty(n)
    L = np.empty(n)
    for p in range(n):
        seg = x[max(p - w, 0):min(p + w, n - 1) + 1]
        U[p], L[p] = seg.max(), seg.min()
    return U, L


def tiles(n, m):
    s = n - m + 1
    out = []
    for L0 in range(m, s, LB_LAGS):
        rows_total = s - L0
        for i0 in range(0, rows_total, LB_ROWS):
            out.append((L0, i0, min(LB_ROWS, rows_total - i0)))
    return out


def upper_profile(x, m, mu, isg):
    """keys of the profile pass: for each row i, the smallest ED^2 over
    j >= i + m truncated to its high 32 bits with the 3 lowest of them
    cleared, and the partner (lowest j on ties); (inf, -1) without a
    partner."""
    s = x.size - m + 1
    W = np.lib.stride_tricks.sliding_window_view(x, m)[:s]
    Z = (W - mu[:, None]) * isg[:, None]
    d2 = np.full(s, np.inf)
    part = np.full(s, -1, dtype=np.int64)
    for i in range(s - m):
        e = ((Z[i + m:] - Z[i]) ** 2).sum(1)
        k = int(np.argmin(e))
        d2[i] = e[k]
        part[i] = i + m + k
    bits = d2.view(np.uint64) & np.uint64(0xFFFFFFF800000000)
    trunc = np.where(np.isfinite(d2), bits.view(np.float64), np.inf)
    return trunc, part


def features(x, m, w):
    """[tiles][64] features in the order of tiles(n, m)."""
    x = np.asarray(x, dtype=np.float64)
    n = x.size
    s = n - m + 1
    mu, isg = stats(x, m)
    U, L = envelope(x, w)
    d2, part = upper_profile(x, m, mu, isg)
    inv = 1.0 / np.sqrt(2.0 * m)
    mpv = np.sqrt(np.maximum(d2, 0.0)) * inv

    def z(i):
        return (x[i:i + m] - mu[i]) * isg[i]

    def fin(v):
        return v if np.isfinite(v) else 4.0

    out = []
    for (L0, i0, rows) in tiles(n, m):
        lags = min(s - 1 - i0 - L0 + 1, LB_LAGS)
        ic = i0 + rows // 2
        Lc = L0 + lags // 2
        if ic + Lc > s - 1:
            Lc = s - 1 - ic
        Lc = max(Lc, m)
        jc = ic + Lc
        f = np.zeros(64)
        zi, zj = z(ic), z(jc)
        for k in range(8):
            a, b = k * m // 8, (k + 1) * m // 8
            f[k] = zi[a:b].mean() if b > a else 0.0
            f[8 + k] = zj[a:b].mean() if b > a else 0.0
        f[16:24] = np.abs(f[0:8] - f[8:16])
        tmin = np.inf
        for k in range(8):
            a, b = k * rows // 8, (k + 1) * rows // 8
            r = np.arange(i0 + a, i0 + b)
            mn = mpv[r].min() if r.size else np.inf
            ok = part[r] >= 0
            lag = part[r] - r
            cnt = np.count_nonzero(ok & (lag >= L0) & (lag < L0 + lags))
            f[24 + k] = fin(mn)
            f[32 + k] = cnt / (b - a) if b > a else 0.0
            tmin = min(tmin, mn)
        for k in range(8):
            r = i0 + (2 * k + 1) * rows // 16
            Lk = min(Lc, s - 1 - r)
            if Lk >= m:
                j = r + Lk
                zr, zc = z(r), z(j)
                u = (U[j:j + m] - mu[j]) * isg[j]
                lo = (L[j:j + m] - mu[j]) * isg[j]
                f[40 + k] = np.sqrt(((zr - zc) ** 2).sum()) * inv
                dd = np.maximum(np.maximum(zr - u, lo - zr), 0.0)
                f[48 + k] = np.sqrt((dd * dd).sum()) * inv
            else:
                f[40 + k] = f[48 + k] = 4.0
        f[56] = L0 / s
        f[57] = i0 / s
        f[58] = rows / LB_ROWS
        f[59] = lags / LB_LAGS
        f[60] = m / 1024.0
        f[61] = w / m
        f[62] = fin(tmin)
        f[63] = 1.0
        out.append(f)
    return np.array(out)
