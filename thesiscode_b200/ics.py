"""Initial vorticity distributions (host side, numpy, FP64).

Two families:
  * the reference's own functions, cited file:line, used for parity runs;
  * the benchmark workloads' formulas (Rossby-Haurwitz wave 4 with
    omega = K = Omega/14, Gaussian vortex exp(-16|x-x0|^2) at 22.5N, the
    sech^2 tanh zonal jet), which differ from the reference's variants in
    sign, amplitude or centre; each function says which it is.
"""
from __future__ import annotations

import numpy as np

PI = np.pi


def atan4(y, x):
    """atan2 with range [0, 2 pi) (SphereGeom.f90:213-248)."""
    t = np.arctan2(y, x)
    return np.where(t < 0.0, t + 2.0 * PI, t)


def longitude(x):
    return atan4(x[..., 1], x[..., 0])


def latitude(x):
    """datan2(z, sqrt(x^2 + y^2)) (SphereGeom.f90:190-195)."""
    return np.arctan2(x[..., 2], np.sqrt(x[..., 0] ** 2 + x[..., 1] ** 2))


def legendre54(z):
    """P_5^4 up to a constant: z (z^2 - 1)^2 (TracerAndVorticityDistributions.f90:459-464)."""
    return z * (-1.0 + z * z) * (-1.0 + z * z)


def rh4_reference(x):
    """HaurwitzStationary4RelVortVector (TracerAndVorticityDistributions.f90:207-217):
    2 (pi/7) z - 30 cc cos(4 lambda) P54(z), cc = -1."""
    alpha_s = PI / 7.0
    cc = -1.0
    return 2.0 * alpha_s * x[..., 2] - 30.0 * cc * np.cos(4.0 * longitude(x)) * legendre54(x[..., 2])


def rh4_config(x, Omega=2.0 * PI):
    """Rossby-Haurwitz wave 4 of the benchmark: 2 w sin(phi) - K sin(phi) cos^4(phi) (4^2+3*4+2)
    cos(4 lambda), w = K = Omega/14; sin(phi) = z, cos^2(phi) = 1 - z^2 on the unit sphere."""
    w = K = Omega / 14.0
    z = x[..., 2]
    c2 = np.clip(1.0 - z * z, 0.0, None)
    return 2.0 * w * z - K * z * c2 * c2 * 30.0 * np.cos(4.0 * longitude(x))


def gaussian_reference(x):
    """GaussianVortexVector (TracerAndVorticityDistributions.f90:398-412): 4 pi exp(-2 b^2 (1 - x.xc)),
    b = 4, centre (lat pi/20, lon 0); the area mean is removed by the caller."""
    lat0, lon0, beta = PI / 20.0, 0.0, 4.0
    xc = np.array([np.cos(lat0) * np.cos(lon0), np.cos(lat0) * np.sin(lon0), np.sin(lat0)])
    return 4.0 * PI * np.exp(-2.0 * beta * beta * (1.0 - x @ xc))


def sphere_point(lat, lon):
    return np.array([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)])


def gaussian_config(x, lat0_deg=22.5, lon0_deg=0.0, beta2=16.0):
    """Benchmark Gaussian vortex exp(-beta2 |x - x0|^2) (beta2 = 16), centre (22.5N, 0E)."""
    x0 = sphere_point(np.deg2rad(lat0_deg), np.deg2rad(lon0_deg))
    d = x - x0
    return np.exp(-beta2 * np.einsum("...c,...c->...", d, d))


def remove_area_mean(zeta_panels, area_panels):
    """gaussConst = sum(g A)/(4 pi) (TracerAndVorticityDistributions.f90:259): the solvability
    condition sum(zeta A) = 0 on the sphere. Returns the constant."""
    return float(np.sum(zeta_panels * area_panels) / (4.0 * PI))


def jet_config(x, U=1.0, phi0=PI / 4.0, width=0.1):
    """Benchmark zonal jet: -U sech^2((phi - phi0)/w) tanh((phi - phi0)/w) / w (U = 1)."""
    s = (latitude(x) - phi0) / width
    return -U * np.tanh(s) / np.cosh(s) ** 2 / width


def jet_reference(x, theta0=PI / 4.0, beta=12.0, perturb_amp=0.025, perturb_wavenum=12):
    """JetRelVortVector (TracerAndVorticityDistributions.f90:829-859) with JetPanels.namelist values."""
    lat = latitude(x)
    lon = longitude(x)
    theta_p = theta0 + perturb_amp * np.cos(perturb_wavenum * lon)
    return 300.0 * np.sin(lat - theta_p) * np.exp(-2.0 * beta * beta * (1.0 - np.cos(lat - theta_p)))


def stratosphere_rel_vort(x, beta=1.5, th0=15.0 * PI / 32.0):
    """StratosphereRelVortX (TracerAndVorticityDistributions.f90:1203-1211): the polar-vortex
    relative vorticity of the forced stratosphere model (before the Gauss constant is removed)."""
    lat = latitude(x)
    return -PI * (np.cos(lat) * (-2.0 * beta * beta * (np.cos(th0) * np.sin(lat) - np.sin(th0) * np.cos(lat)))
                  - np.sin(lat)) * np.exp(-2.0 * beta * beta * (1.0 - np.cos(th0) * np.cos(lat)
                                                                 - np.sin(th0) * np.sin(lat)))


def solid_body(x, rotation_rate):
    """InitSolidBody / SolidBodyX (TracerAndVorticityDistributions.f90:1246-1268): 2 w z.
    With Omega = 0 the exact velocity is u = w z_hat x x (solidBody.f90:296-300)."""
    return 2.0 * rotation_rate * x[..., 2]
