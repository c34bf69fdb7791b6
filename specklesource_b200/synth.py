"""Seeded synthetic SAR pairs (the benchmark and test inputs).

No public dataset is involved: every workload is a circular-Gaussian speckle
field, band-limited to 0.8 of the spectrum per axis, resampled by a known
displacement field with a 16-tap Kaiser-windowed sinc (beta = 6), mixed with
independent speckle for a chosen coherence and multiplied by a range phase
ramp.  Generation uses torch so the large pairs can be built on the GPU;
results are complex64 (na, nr) arrays.
"""
import math

import numpy as np
import torch

TAPS = 16
KAISER_BETA = 6.0


def _speckle(na, nr, gen, device, band=0.8):
    z = torch.complex(torch.randn(na, nr, generator=gen, device=device),
                      torch.randn(na, nr, generator=gen, device=device))
    Z = torch.fft.fft2(z)
    fy = torch.fft.fftfreq(na, device=device).abs() <= band / 2
    fx = torch.fft.fftfreq(nr, device=device).abs() <= band / 2
    Z = Z * (fy[:, None] & fx[None, :])
    z = torch.fft.ifft2(Z)
    z = z / torch.sqrt((z.abs() ** 2).mean())
    return z.to(torch.complex64)


def _sinc_kernel(frac):
    """Windowed-sinc weights (..., TAPS) for fractional offsets in [0,1)."""
    t = torch.arange(TAPS, device=frac.device, dtype=torch.float64) - (TAPS // 2 - 1)
    x = t - frac[..., None].double()
    w = torch.special.i0(KAISER_BETA * torch.sqrt(torch.clamp(1 - (x / (TAPS / 2)) ** 2, min=0.0)))
    w = w / torch.special.i0(torch.tensor(KAISER_BETA, dtype=torch.float64, device=frac.device))
    h = torch.sinc(x) * w
    return h / h.sum(-1, keepdim=True)


def _resample_axis(z, shift, axis, chunk=1 << 22):
    """out[..., x] = z[..., x + shift[..., x]] along `axis` (1 = range, 0 = azimuth)."""
    if axis == 0:
        return _resample_axis(z.T.contiguous(), shift.T.contiguous(), 1, chunk).T.contiguous()
    na, nr = z.shape
    out = torch.empty_like(z)
    rows_per = max(1, chunk // nr)
    xs = torch.arange(nr, device=z.device, dtype=torch.float64)
    for r0 in range(0, na, rows_per):
        r1 = min(na, r0 + rows_per)
        pos = xs[None, :] + shift[r0:r1].double()
        base = torch.floor(pos)
        frac = pos - base
        h = _sinc_kernel(frac).to(torch.float32)  # (rows, nr, TAPS)
        idx = base.long()[..., None] + torch.arange(TAPS, device=z.device) - (TAPS // 2 - 1)
        idx = idx.clamp(0, nr - 1)
        src = z[r0:r1]
        g = torch.gather(src, 1, idx.reshape(r1 - r0, -1)).reshape(r1 - r0, nr, TAPS)
        out[r0:r1] = (g * h).sum(-1)
    return out


def make_pair(na, nr, seed, dr, da, coherence=0.7, ramp=0.01, device="cpu"):
    """Reference/secondary pair.

    dr, da: callables (yy, xx) -> displacement (pixels) in range / azimuth,
    evaluated on float64 grids of image coordinates.  coherence: scalar or
    callable (yy, xx) -> gamma.  Returns (img1, img2) complex64 torch tensors.
    """
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    s1 = _speckle(na, nr, gen, device)
    noise = _speckle(na, nr, gen, device)
    yy = torch.arange(na, device=device, dtype=torch.float64)[:, None].expand(na, nr)
    xx = torch.arange(nr, device=device, dtype=torch.float64)[None, :].expand(na, nr)
    sr = dr(yy, xx).to(torch.float32)
    sa = da(yy, xx).to(torch.float32)
    # s2(y, x) = s1(y - da, x - dr): a feature at x in image 1 sits at x + dr
    # in image 2, so the tracked offsets equal (dr, da).
    res = _resample_axis(s1, -sr, 1)
    res = _resample_axis(res, -sa, 0)
    g = coherence(yy, xx).to(torch.float32) if callable(coherence) else torch.full(
        (na, nr), float(coherence), device=device)
    s2 = g * res + torch.sqrt(1 - g * g) * noise
    s2 = s2 * torch.exp(1j * ramp * xx.to(torch.float32))
    return s1, s2.to(torch.complex64)


# ---------------------------------------------------------------------------
# The workloads (stand-ins for the benchmark configurations)
# ---------------------------------------------------------------------------


def small_pair(device="cpu", na=1024, nr=2048, seed=1):
    """1024 az x 2048 rg pair: rg shift 2+1.5 sin(2 pi x/1500), az shift
    0.5 cos(2 pi y/900), coherence 0.7, ramp 0.01 rad/px."""
    return make_pair(na, nr, seed,
                     dr=lambda y, x: 2 + 1.5 * torch.sin(2 * math.pi * x / 1500),
                     da=lambda y, x: 0.5 * torch.cos(2 * math.pi * y / 900),
                     coherence=0.7, device=device)


def large_pair(device="cuda", na=12000, nr=24000, seed=2):
    """12000 x 24000 pair: coherence per 512-px block uniform in [0.3, 0.9],
    smooth displacement within +-12 px (range) and +-4 px (azimuth)."""
    gen = torch.Generator(device="cpu")
    gen.manual_seed(seed + 1000)
    nby, nbx = (na + 511) // 512, (nr + 511) // 512
    blocks = (0.3 + 0.6 * torch.rand(nby, nbx, generator=gen, dtype=torch.float64)).to(device)

    def coh(y, x):
        return blocks[(y // 512).long(), (x // 512).long()]

    return make_pair(na, nr, seed,
                     dr=lambda y, x: 12 * torch.sin(2 * math.pi * x / 9000) * torch.cos(2 * math.pi * y / 7000),
                     da=lambda y, x: 4 * torch.cos(2 * math.pi * (x + y) / 11000),
                     coherence=coh, device=device)


def shear_pair(device="cuda", na=8000, nr=16000, seed=3):
    """Fast-flow pair: a diagonal shear zone with |d| <= 40 px, coherence in
    [0.25, 0.5] varying smoothly."""
    def dr(y, x):
        s = (x - 2 * y) / 1500.0
        return 40 * torch.tanh(s)

    def da(y, x):
        s = (x - 2 * y) / 1500.0
        return 10 * torch.tanh(s)

    def coh(y, x):
        return 0.375 + 0.125 * torch.sin(2 * math.pi * x / 5000) * torch.cos(2 * math.pi * y / 3000)

    return make_pair(na, nr, seed, dr=dr, da=da, coherence=coh, device=device)


def to_numpy(t):
    return t.detach().cpu().numpy()


def to_big_endian(a):
    """complex64 array -> big-endian '>c8' array (the on-disk SLC format)."""
    return np.ascontiguousarray(a).astype(">c8")


_LARGE = np.float32(-2e9)


def offsets_field(nA, nR, seed, outliers=0.08, holes=0.02):
    """Smooth offsets with uniform +-20 px outliers, NaN holes and failed points."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:nA, 0:nR].astype(np.float64)
    offR = 3 + 2 * np.sin(xx / 37.0) * np.cos(yy / 23.0) + 0.05 * rng.standard_normal((nA, nR))
    offA = -1 + np.cos((xx + yy) / 41.0) + 0.05 * rng.standard_normal((nA, nR))
    m = rng.random((nA, nR)) < outliers
    offR[m] += rng.uniform(-20, 20, m.sum())
    offA[m] += rng.uniform(-20, 20, m.sum())
    h = rng.random((nA, nR)) < holes
    offR[h] = np.nan
    offA[h] = np.nan
    f = rng.random((nA, nR)) < 0.05
    offR[f] = _LARGE
    offA[f] = _LARGE
    # a failed region holding small valid islands (they survive the median
    # passes and are removed by the island pass) and one larger valid patch
    a0, r0 = nA // 5, nR // 5
    block = (slice(a0, a0 + 60), slice(r0, r0 + 90))
    offR[block] = _LARGE
    offA[block] = _LARGE
    f[block] = True
    for k, (di, dj, s) in enumerate([(5, 5, 8), (5, 40, 7), (30, 10, 9), (30, 50, 25)]):
        isl = (slice(a0 + di, a0 + di + s), slice(r0 + dj, r0 + dj + min(s, 35)))
        offR[isl] = 3.0 + 0.01 * k
        offA[isl] = -1.0
        f[isl] = False
    corr = rng.uniform(0, 1, (nA, nR)).astype(np.float32)
    mt = rng.integers(1, 4, (nA, nR)).astype(np.uint8)
    mt[f] = 0
    return offR.astype(np.float32), offA.astype(np.float32), corr, mt


def fringe_interferogram(na, nr, nrl, nal, ramp_r, ramp_a=0.0, amp=1000.0, byte_order=">"):
    """Multi-looked interferogram of a linear fringe, as getInt reads it:
    complex int16 (re, im) samples, (na // nal) x (nr // nrl), sample (i, k)
    covering SLC rows i*nal.. and columns k*nrl..; phase -(ramp_r x + ramp_a y)
    at its first pixel, the phase of s1 conj(s2) for a pair whose secondary
    image carries exp(+i (ramp_r x + ramp_a y)).  The fringe must stay below
    pi per look (|ramp_r| nrl, |ramp_a| nal < pi) to be representable."""
    ia = np.arange(na // nal)[:, None] * nal
    ir = np.arange(nr // nrl)[None, :] * nrl
    ph = -(ramp_r * ir + ramp_a * ia)
    out = np.empty((na // nal, nr // nrl, 2), np.float64)
    out[..., 0] = amp * np.cos(ph)
    out[..., 1] = amp * np.sin(ph)
    return np.round(out).astype(byte_order + "i2")
