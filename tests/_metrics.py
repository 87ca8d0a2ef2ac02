"""Image-comparison metrics used by the parity tests.

The headline metric is the per-pixel relative error of the composited
linear-HDR image `hdr = L + background * T` (what the reference writes into
its HDR target), max over RGB, against the FP64 oracle.  The background is a
smooth positive sky, so the denominator never vanishes.
"""
import numpy as np


def composite(L, T, bg):
    return L + bg * T


def rel_stats(a, b):
    """Stats of max-over-RGB |a-b|/|b| per pixel."""
    r = (np.abs(a[..., :3] - b[..., :3]) / np.maximum(np.abs(b[..., :3]), 1e-30)).max(-1).ravel()
    return {"max": float(r.max()), "p999": float(np.quantile(r, 0.999)),
            "p99": float(np.quantile(r, 0.99)), "mean": float(r.mean()),
            "frac_gt_1e3": float((r > 1e-3).mean())}


def tonemap(hdr, exposure=1.0 / 12000.0):
    """Reinhard on exposed luminance-scaled RGB, then sRGB-ish gamma; [0,1]."""
    x = np.maximum(hdr[..., :3] * exposure, 0)
    return (x / (1.0 + x)) ** (1 / 2.2)


def ssim(a, b):
    """Mean SSIM over channels (Gaussian window sigma 1.5, as Wang et al. 2004)."""
    from scipy.ndimage import gaussian_filter
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    vals = []
    for ch in range(a.shape[-1]):
        x, y = a[..., ch].astype(np.float64), b[..., ch].astype(np.float64)
        mx, my = gaussian_filter(x, 1.5), gaussian_filter(y, 1.5)
        sxx = gaussian_filter(x * x, 1.5) - mx * mx
        syy = gaussian_filter(y * y, 1.5) - my * my
        sxy = gaussian_filter(x * y, 1.5) - mx * my
        m = ((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))
        vals.append(m.mean())
    return float(np.mean(vals))
