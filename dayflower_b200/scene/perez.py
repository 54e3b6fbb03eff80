"""Host-side precompute of the Perez sun-and-sky light record.

Restates what ``scene/light/PerezLight.java`` computes when the light is set up
(``set(turbidity, sunDirectionWorldSpace)``) and what
``scene/compiler/CompiledLightCache.java:1495`` (``toPerezLight``) stores:

* the fixed sky transform (object z is world y), ``doSetTransform``;
* the sun direction in both spaces and its zenith angle ``theta``;
* the Preetham zenith luminance/chromaticity, ``doSetZenith``;
* the attenuated sun colour, ``doSetSunColor`` / ``doCalculateAttenuatedSunlight``;
* the 32x32 luminance distribution for importance sampling,
  ``doInitializeDistribution`` packed by ``sampler/Distribution2F.toArray``.

The spectral tables are the published Preetham-Shirley-Smits (1999) daylight
data the reference also uses.  The spectrum-to-XYZ step integrates against the
multi-lobe analytic fit of the CIE 1931 matching functions by Wyman, Sloan and
Shirley (2013) instead of the tabulated functions; the result is an input value
of the compiled scene, consumed as given by the renderer and the oracle alike.
"""
from __future__ import annotations

import math

import numpy as np

# Preetham et al. absorption coefficients and solar spectral radiance.
_K_O_WL = [300, 305, 310, 315, 320, 325, 330, 335, 340, 345, 350, 355, 445, 450, 455, 460, 465, 470, 475, 480, 485, 490, 495,
           500, 505, 510, 515, 520, 525, 530, 535, 540, 545, 550, 555, 560, 565, 570, 575, 580, 585, 590, 595, 600, 605, 610,
           620, 630, 640, 650, 660, 670, 680, 690, 700, 710, 720, 730, 740, 750, 760, 770, 780, 790]
_K_O_AMP = [10.0, 4.8, 2.7, 1.35, 0.8, 0.380, 0.160, 0.075, 0.04, 0.019, 0.007, 0.0, 0.003, 0.003, 0.004, 0.006, 0.008, 0.009,
            0.012, 0.014, 0.017, 0.021, 0.025, 0.03, 0.035, 0.04, 0.045, 0.048, 0.057, 0.063, 0.07, 0.075, 0.08, 0.085, 0.095,
            0.103, 0.110, 0.12, 0.122, 0.12, 0.118, 0.115, 0.12, 0.125, 0.130, 0.12, 0.105, 0.09, 0.079, 0.067, 0.057, 0.048,
            0.036, 0.028, 0.023, 0.018, 0.014, 0.011, 0.010, 0.009, 0.007, 0.004, 0.0, 0.0]
_K_G_WL = [759, 760, 770, 771]
_K_G_AMP = [0.0, 3.0, 0.210, 0.0]
_K_WA_WL = [689, 690, 700, 710, 720, 730, 740, 750, 760, 770, 780, 790, 800]
_K_WA_AMP = [0.0, 0.160e-1, 0.240e-1, 0.125e-1, 0.100e+1, 0.870, 0.610e-1, 0.100e-2, 0.100e-4, 0.100e-4, 0.600e-3, 0.175e-1,
             0.360e-1]
_SOL_AMP = [165.5, 162.3, 211.2, 258.8, 258.2, 242.3, 267.6, 296.6, 305.4, 300.6, 306.6, 288.3, 287.1, 278.2, 271.0, 272.3,
            263.6, 255.0, 250.6, 253.1, 253.5, 251.3, 246.3, 241.7, 236.8, 232.1, 228.2, 223.4, 219.7, 215.3, 211.0, 207.3,
            202.4, 198.7, 194.3, 190.7, 186.3, 182.6]  # 380..750 nm, regular


def _irregular(wl, amp, lam):
    """``IrregularSpectralCurveF.sample``: clamp below, linear inside, clamp above."""
    if lam <= wl[0]:
        return amp[0]
    for i in range(1, len(wl)):
        if lam < wl[i]:
            d = (lam - wl[i - 1]) / (wl[i] - wl[i - 1])
            return (1.0 - d) * amp[i - 1] + d * amp[i]
    return amp[-1]


def _regular(lo, hi, spec, lam):
    """``RegularSpectralCurveF.sample``: zero outside [lo, hi], linear inside."""
    if lam < lo or lam > hi:
        return 0.0
    x = (lam - lo) * ((len(spec) - 1) / (hi - lo))
    i0 = int(x)
    i1 = min(i0 + 1, len(spec) - 1)
    d = x - i0
    return (1.0 - d) * spec[i0] + d * spec[i1]


def _cie_xyz_fit(lam: np.ndarray):
    """Wyman-Sloan-Shirley (2013) multi-lobe fit of the CIE 1931 2-degree observer."""
    def g(x, mu, s1, s2):
        s = np.where(x < mu, s1, s2)
        return np.exp(-0.5 * ((x - mu) * s) ** 2)
    x = 1.056 * g(lam, 599.8, 0.0264, 0.0323) + 0.362 * g(lam, 442.0, 0.0624, 0.0374) - 0.065 * g(lam, 501.1, 0.0490, 0.0382)
    y = 0.821 * g(lam, 568.8, 0.0213, 0.0247) + 0.286 * g(lam, 530.9, 0.0613, 0.0322)
    z = 1.217 * g(lam, 437.0, 0.0845, 0.0278) + 0.681 * g(lam, 459.0, 0.0385, 0.0725)
    return x, y, z


def _spectrum_to_xyz(lo, hi, spec):
    """``SpectralCurveF.toColorXYZ`` over 360..830 nm in 1 nm steps."""
    lam = np.arange(360.0, 831.0, 1.0)
    s = np.array([_regular(lo, hi, spec, float(l)) for l in lam])
    xb, yb, zb = _cie_xyz_fit(lam)
    y_integral = float(np.sum(yb))
    scale = (lam[-1] - lam[0]) / (y_integral * len(lam))
    return np.array([np.sum(s * xb), np.sum(s * yb), np.sum(s * zb)]) * scale


def _sun_spectrum(theta: float, turbidity: float):
    """``PerezLight.doCalculateAttenuatedSunlight``: 350..800 nm in 5 nm steps."""
    alpha, lozone, w = 1.3, 0.35, 2.0
    beta = 0.04608365822050 * turbidity - 0.04586025928522
    m = 1.0 / (math.cos(theta) + 0.000940 * math.pow(1.6386 - theta, -1.253))
    out = []
    for lam in range(350, 801, 5):
        tr = math.exp(-m * 0.008735 * math.pow(lam / 1000.0, -4.08))
        ta = math.exp(-m * beta * math.pow(lam / 1000.0, -alpha))
        to = math.exp(-m * _irregular(_K_O_WL, _K_O_AMP, lam) * lozone)
        kg = _irregular(_K_G_WL, _K_G_AMP, lam)
        tg = math.exp(-1.41 * kg * m / math.pow(1.0 + 118.93 * kg * m, 0.45))
        kwa = _irregular(_K_WA_WL, _K_WA_AMP, lam)
        twa = math.exp(-0.2385 * kwa * w * m / math.pow(1.0 + 20.07 * kwa * w * m, 0.45))
        out.append(np.float32(_regular(380.0, 750.0, _SOL_AMP, lam) * tr * ta * to * tg * twa))
    return out


# sRGB (color/ColorSpaceF.java:85) XYZ->RGB matrix derived from the primaries.
def _xyz_to_rgb_matrix():
    xr, yr, xg, yg, xb, yb, xw, yw = 0.64, 0.33, 0.3, 0.6, 0.15, 0.06, 0.31271, 0.32902
    zr, zg, zb, zw = 1 - (xr + yr), 1 - (xg + yg), 1 - (xb + yb), 1 - (xw + yw)
    rx, ry, rz = yg * zb - yb * zg, xb * zg - xg * zb, xg * yb - xb * yg
    gx, gy, gz = yb * zr - yr * zb, xr * zb - xb * zr, xb * yr - xr * yb
    bx, by, bz = yr * zg - yg * zr, xg * zr - xr * zg, xr * yg - xg * yr
    rw = (rx * xw + ry * yw + rz * zw) / yw
    gw = (gx * xw + gy * yw + gz * zw) / yw
    bw = (bx * xw + by * yw + bz * zw) / yw
    return np.array([[rx / rw, ry / rw, rz / rw], [gx / gw, gy / gw, gz / gw], [bx / bw, by / bw, bz / bw]])


_XYZ2RGB = _xyz_to_rgb_matrix()

# Sky transform: Matrix44F.rotate(OrthonormalBasis33F(w = y, v = x)) has columns (u, v, w) = (z, x, y).
SKY_OBJECT_TO_WORLD = np.array([[0, 1, 0, 0], [0, 0, 1, 0], [1, 0, 0, 0], [0, 0, 0, 1]], dtype=np.float32)
SKY_WORLD_TO_OBJECT = SKY_OBJECT_TO_WORLD.T.copy()


def _perez(lam, theta, gamma, lvz, theta_s):
    den = (1.0 + lam[0] * math.exp(lam[1])) * (1.0 + lam[2] * math.exp(lam[3] * theta_s) + lam[4] * math.cos(theta_s) ** 2)
    num = (1.0 + lam[0] * math.exp(lam[1] / math.cos(theta))) * (1.0 + lam[2] * math.exp(lam[3] * gamma) + lam[4] * math.cos(gamma) ** 2)
    return lvz * num / den


def _sky_rgb(direction, sun_obj, T, zenith, theta_s):
    """``PerezLight.doRadianceSky`` in double precision (host side)."""
    d = np.asarray(direction, dtype=np.float64)
    if d[2] < 0.0:
        return np.zeros(3)
    d = np.array([d[0], d[1], max(d[2], 0.001)])
    d /= np.linalg.norm(d)
    theta = math.acos(min(max(d[2], -1.0), 1.0))
    gamma = math.acos(min(max(float(np.dot(d, sun_obj)), -1.0), 1.0))
    pl = [0.17872 * T - 1.46303, -0.35540 * T + 0.42749, -0.02266 * T + 5.32505, 0.12064 * T - 2.57705, -0.06696 * T + 0.37027]
    px = [-0.01925 * T - 0.25922, -0.06651 * T + 0.00081, -0.00041 * T + 0.21247, -0.06409 * T - 0.89887, -0.00325 * T + 0.04517]
    py = [-0.01669 * T - 0.26078, -0.09495 * T + 0.00921, -0.00792 * T + 0.21023, -0.04405 * T - 1.65369, -0.01092 * T + 0.05291]
    Y = _perez(pl, theta, gamma, zenith[0], theta_s) * 0.0001
    x = _perez(px, theta, gamma, zenith[1], theta_s)
    y = _perez(py, theta, gamma, zenith[2], theta_s)
    m1 = (-1.3515 - 1.7703 * x + 5.9114 * y) / (0.0241 + 0.2562 * x - 0.7341 * y)
    m2 = (0.03 - 31.4424 * x + 30.0717 * y) / (0.0241 + 0.2562 * x - 0.7341 * y)
    X = 95.6824722290 + m1 * 1.7548348904 + m2 * 1.9917192459
    Yc = 99.7036819458 + m1 * 1.8025954962 + m2 * 0.7136800885
    Z = 115.5248031616 + m1 * 32.5218048096 + m2 * -2.1984319687
    return _XYZ2RGB @ np.array([X * Y / Yc, Y, Z * Y / Yc])


def _distribution1(func):
    """``Distribution1F`` constructor + ``toArray``."""
    f = np.asarray(func, dtype=np.float32)
    n = len(f)
    cdf = np.zeros(n + 1, dtype=np.float32)
    for i in range(1, n + 1):
        cdf[i] = np.float32(cdf[i - 1] + np.float32(f[i - 1] / np.float32(n)))
    integral = np.float32(cdf[n])
    if integral == 0.0:
        cdf = (np.arange(n + 1) / n).astype(np.float32)
    else:
        cdf[1:] = (cdf[1:] / integral).astype(np.float32)
    arr = np.zeros(4 + (n + 1) + n, dtype=np.float32)
    arr[0] = len(arr)
    arr[1] = n + 1
    arr[2] = n
    arr[3] = integral
    arr[4:4 + n + 1] = cdf
    arr[4 + n + 1:] = f
    return arr, integral


def _distribution2_uv(functions):
    """``Distribution2F(functions, isUV = true).toArray()``."""
    conds, integrals = [], []
    for row in functions:
        a, integ = _distribution1(row)
        conds.append(a)
        integrals.append(integ)
    marg, _ = _distribution1(integrals)
    m = len(functions)
    offsets = np.zeros(1 + m, dtype=np.float32)
    offsets[0] = len(offsets) + 1 + 1
    for i in range(m):
        offsets[i + 1] = int(offsets[i]) + (len(marg) if i == 0 else len(conds[i - 1]))
    return np.concatenate([np.array([1.0, len(offsets)], dtype=np.float32), offsets, marg] + conds).astype(np.float32)


def perez_record(turbidity: float, sun_direction_world) -> np.ndarray:
    """The compiled PerezLight record (``CompiledLightCache.toPerezLight``), padded to 8."""
    T = float(turbidity)
    sun_w = np.asarray(sun_direction_world, dtype=np.float64)
    sun_w = sun_w / np.linalg.norm(sun_w)
    sun_o = SKY_WORLD_TO_OBJECT[:3, :3].astype(np.float64) @ sun_w
    sun_o /= np.linalg.norm(sun_o)
    theta = math.acos(min(max(sun_o[2], -1.0), 1.0))
    z0 = ((4.0453 * T - 4.9710) * math.tan((4.0 / 9.0 - T / 120.0) * (math.pi - 2.0 * theta)) - 0.2155 * T + 2.4192) * 1000.0
    t2, t3 = theta * theta, theta * theta * theta
    z1 = (0.00165 * t3 - 0.00374 * t2 + 0.00208 * theta) * T * T + (-0.02902 * t3 + 0.06377 * t2 - 0.03202 * theta + 0.00394) * T + (0.11693 * t3 - 0.21196 * t2 + 0.06052 * theta + 0.25885)
    z2 = (0.00275 * t3 - 0.00610 * t2 + 0.00316 * theta) * T * T + (-0.04212 * t3 + 0.08970 * t2 - 0.04153 * theta + 0.00515) * T + (0.15346 * t3 - 0.26756 * t2 + 0.06669 * theta + 0.26688)
    zenith = (z0, z1, z2)
    if sun_o[2] > 0.0:
        xyz = _spectrum_to_xyz(350.0, 800.0, _sun_spectrum(theta, T)) * 0.0001
        sun_color = np.maximum(_XYZ2RGB @ xyz, 0.0)
    else:
        sun_color = np.zeros(3)
    funcs = np.zeros((32, 32), dtype=np.float32)
    for u in range(32):
        su = (u + 0.5) / 32.0
        for v in range(32):
            sv = (v + 0.5) / 32.0
            phi, th = su * 2.0 * math.pi, sv * math.pi
            d = (math.sin(th) * math.cos(phi), math.sin(th) * math.sin(phi), math.cos(th))
            rgb = np.maximum(_sky_rgb(d, sun_o, T, zenith, theta), 0.0)
            lum = rgb[0] * 0.212671 + rgb[1] * 0.715160 + rgb[2] * 0.072169
            funcs[u, v] = np.float32(lum * math.sin(math.pi * sv))
    dist = _distribution2_uv(funcs)
    head = np.zeros(48, dtype=np.float32)
    head[0:16] = SKY_OBJECT_TO_WORLD.reshape(-1)
    head[16:32] = SKY_WORLD_TO_OBJECT.reshape(-1)
    head[32:35] = sun_color
    head[35:38] = sun_o
    head[38:41] = sun_w
    head[41] = T
    head[42:45] = zenith
    head[45] = 10.0  # doSetRadius
    head[46] = theta
    rec = np.concatenate([head, dist])
    pad = (-len(rec)) % 8
    return np.concatenate([rec, np.zeros(pad, dtype=np.float32)]).astype(np.float32)


# ---- ImageLight ------------------------------------------------------------------
def image_sky_rgb(image: np.ndarray, angle_rad: float, scale, dirs: np.ndarray) -> np.ndarray:
    """``ImageLight.doRadianceSky`` for object-space unit directions (n, 3):
    spherical texture coordinates (Point2F.sphericalCoordinates), rotated
    counterclockwise, scaled, mapped to pixel space (Point2F.toImage) and looked
    up with bilinear interpolation and wrap-around (ImageF.getColorRGB)."""
    f32 = np.float32
    h, w = image.shape[0], image.shape[1]
    d = dirs.astype(np.float32)
    phi = np.arctan2(d[:, 1].astype(np.float64), d[:, 0].astype(np.float64)).astype(f32)
    phi = np.where(phi < 0, phi + f32(2.0 * math.pi), phi).astype(f32)
    theta = np.arccos(np.clip(d[:, 2], -1.0, 1.0)).astype(f32)
    u = (phi * f32(1.0 / (2.0 * math.pi))).astype(f32)
    v = (theta * f32(1.0 / math.pi)).astype(f32)
    c, s_ = f32(math.cos(angle_rad)), f32(math.sin(angle_rad))
    ur = (u * c - v * s_).astype(f32)
    vr = (v * c + u * s_).astype(f32)
    us, vs = (ur * f32(scale[0])).astype(f32), (vr * f32(scale[1])).astype(f32)

    def posmod(x, y):
        return np.where(x < 0, np.fmod(np.fmod(x, y) + y, y), np.fmod(x, y)).astype(f32)

    x = posmod((us * f32(w) - f32(0.5)).astype(f32), f32(w))
    y = posmod((vs * f32(h) - f32(0.5)).astype(f32), f32(h))
    x0, x1 = np.floor(x).astype(np.int64), np.ceil(x).astype(np.int64)
    y0, y1 = np.floor(y).astype(np.int64), np.ceil(y).astype(np.int64)
    xf, yf = (x - x0).astype(f32)[:, None], (y - y0).astype(f32)[:, None]
    c00 = image[y0 % h, x0 % w]
    c01 = image[y0 % h, x1 % w]
    c10 = image[y1 % h, x0 % w]
    c11 = image[y1 % h, x1 % w]
    top = (1 - xf) * c00 + xf * c01
    bot = (1 - xf) * c10 + xf * c11
    return ((1 - yf) * top + yf * bot).astype(f32)


def image_light_record(image: np.ndarray, angle_deg: float = 0.0, scale=(1.0, 1.0)) -> np.ndarray:
    """The compiled ImageLight record (``CompiledLightCache.toImageLight``,
    CompiledLightCache.java:1393-1460): object-to-world and world-to-object
    matrices, angle, scale, radius 10, resolution, the 32x32 luminance
    distribution of ``ImageLight.doCreateDistribution`` and the RGB image."""
    img = np.ascontiguousarray(image, dtype=np.float32)
    h, w = img.shape[0], img.shape[1]
    ang = math.radians(angle_deg)
    su = (np.arange(32, dtype=np.float32) + np.float32(0.5)) * np.float32(1.0 / 32.0)
    U, V = np.meshgrid(su, su, indexing="ij")  # functions[u][v]
    phi, th = U * np.float32(2.0 * math.pi), V * np.float32(math.pi)
    d = np.stack([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.cos(th)], axis=-1).reshape(-1, 3).astype(np.float32)
    rgb = image_sky_rgb(img, ang, scale, d)
    lum = rgb[:, 0] * np.float32(0.212671) + rgb[:, 1] * np.float32(0.715160) + rgb[:, 2] * np.float32(0.072169)
    funcs = (lum.reshape(32, 32) * np.sin(np.float32(math.pi) * V)).astype(np.float32)
    dist = _distribution2_uv(funcs)
    head = np.zeros(40, dtype=np.float32)
    head[0:16] = SKY_OBJECT_TO_WORLD.reshape(-1)
    head[16:32] = SKY_WORLD_TO_OBJECT.reshape(-1)
    head[32] = ang
    head[33], head[34] = scale
    head[35] = 10.0  # ImageLight radius
    head[36], head[37] = w, h
    assert len(dist) == 2312
    rec = np.concatenate([head, dist, img.reshape(-1)])
    pad = (-len(rec)) % 8
    return np.concatenate([rec, np.zeros(pad, dtype=np.float32)]).astype(np.float32)
