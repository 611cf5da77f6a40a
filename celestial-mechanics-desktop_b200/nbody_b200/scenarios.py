"""Seeded initial conditions for the force-path workloads.

The reference draws its scenarios from .NET ``System.Random``
(src/CelestialMechanics.Physics/ScenarioGenerators/PlummerSphere.cs:44), whose
stream cannot be reproduced without .NET.  These generators restate the same
sampling algorithms on numpy's PCG64 so that every implementation (engine,
oracle, reference CPU code) is fed the very same arrays.

Units: G = 1, AU, solar masses (engine/include/celestial/core/constants.hpp:26).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

#: 3 g/cm^3 in solar masses per cubic AU.
DENSITY_3GCC_MSUN_AU3 = 3000.0 * (1.495978707e11 ** 3) / 1.98847e30


@dataclass
class Bodies:
    """Host structure-of-arrays, the fields of BodySoA
    (src/CelestialMechanics.Physics/SoA/BodySoA.cs:39-175) the force path uses."""

    px: np.ndarray
    py: np.ndarray
    pz: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    mass: np.ndarray
    radius: np.ndarray
    active: np.ndarray
    density: np.ndarray | None = None
    collidable: np.ndarray | None = None
    ax: np.ndarray = field(default=None)
    ay: np.ndarray = field(default=None)
    az: np.ndarray = field(default=None)

    def __post_init__(self):
        n = len(self.px)
        for name in ("ax", "ay", "az"):
            if getattr(self, name) is None:
                setattr(self, name, np.zeros(n))

    @property
    def n(self) -> int:
        return len(self.px)

    def copy(self) -> "Bodies":
        kw = {k: (None if v is None else v.copy()) for k, v in self.__dict__.items()}
        return Bodies(**kw)


def _dirs(rng: np.random.Generator, n: int):
    cos_t = 2.0 * rng.random(n) - 1.0
    sin_t = np.sqrt(1.0 - cos_t * cos_t)
    phi = 2.0 * np.pi * rng.random(n)
    return sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t


def plummer(n: int, total_mass: float = 1.0, scale: float = 1.0, seed: int = 0) -> Bodies:
    """Plummer sphere with Aarseth-Henon-Wielen sampling, as PlummerSphere.Generate
    (PlummerSphere.cs:41-117): inverse-CDF radius with u clamped to
    [1e-10, 1-1e-10], isotropic direction, speed q*v_esc(r) with q drawn by
    rejection from q^2 (1-q^2)^(7/2) under the envelope 0.1."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = np.clip(rng.random(n), 1e-10, 1.0 - 1e-10)
    r = scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    dx, dy, dz = _dirs(rng, n)
    v_esc = np.sqrt(2.0 * total_mass / np.sqrt(r * r + scale * scale))
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        qq = rng.random(todo.size)
        g = qq * qq * (1.0 - qq * qq) ** 3.5
        ok = rng.random(todo.size) * 0.1 < g
        q[todo[ok]] = qq[ok]
        todo = todo[~ok]
    speed = q * v_esc
    ex, ey, ez = _dirs(rng, n)
    return Bodies(px=r * dx, py=r * dy, pz=r * dz, vx=speed * ex, vy=speed * ey, vz=speed * ez,
                  mass=np.full(n, total_mass / n), radius=np.full(n, 0.02),
                  active=np.ones(n, np.uint8))


def _hernquist_df(e_bind: np.ndarray, total_mass: float, scale: float) -> np.ndarray:
    """Isotropic Hernquist distribution function f(E) (Hernquist 1990, ApJ 356,
    359, eq. 17) as a function of the binding energy E > 0 (G = 1)."""
    q = np.sqrt(np.clip(e_bind * scale / total_mass, 0.0, 1.0 - 1e-15))
    vg = np.sqrt(total_mass / scale)
    pref = total_mass / (8.0 * np.sqrt(2.0) * np.pi ** 3 * scale ** 3 * vg ** 3)
    q2 = q * q
    return pref / (1.0 - q2) ** 2.5 * (3.0 * np.arcsin(q) + q * np.sqrt(1.0 - q2) * (1.0 - 2.0 * q2)
                                      * (8.0 * q2 * q2 - 8.0 * q2 - 3.0))


def hernquist(n: int, total_mass: float = 1.0, scale: float = 1.0, seed: int = 4,
              r_max_frac: float = 0.999) -> Bodies:
    """Hernquist sphere (Hernquist 1990): r = a sqrt(U) / (1 - sqrt(U)) with U
    capped at r_max_frac of the mass, speeds by rejection from
    v^2 f(Psi(r) - v^2/2) on [0, v_esc], isotropic directions."""
    rng = np.random.Generator(np.random.PCG64(seed))
    s = np.sqrt(rng.random(n) * r_max_frac)
    r = scale * s / (1.0 - s)
    dx, dy, dz = _dirs(rng, n)
    psi = total_mass / (r + scale)
    v_esc = np.sqrt(2.0 * psi)
    grid = np.linspace(0.0, 1.0, 65)[1:-1]
    # envelope: 1.2 x the maximum of v^2 f on a 63-point grid, per body
    gmax = np.zeros(n)
    for t in grid:
        v = t * v_esc
        gmax = np.maximum(gmax, v * v * _hernquist_df(psi - 0.5 * v * v, total_mass, scale))
    gmax *= 1.2
    speed = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        v = rng.random(todo.size) * v_esc[todo]
        g = v * v * _hernquist_df(psi[todo] - 0.5 * v * v, total_mass, scale)
        ok = rng.random(todo.size) * gmax[todo] < g
        speed[todo[ok]] = v[ok]
        todo = todo[~ok]
    ex, ey, ez = _dirs(rng, n)
    return Bodies(px=r * dx, py=r * dy, pz=r * dz, vx=speed * ex, vy=speed * ey,
                  vz=speed * ez, mass=np.full(n, total_mass / n), radius=np.full(n, 0.02),
                  active=np.ones(n, np.uint8))


def _kepler_state(a, e, inc, node, peri, mean_anom, mu):
    """Cartesian state from orbital elements (Newton iteration on Kepler's equation)."""
    E = mean_anom.copy()
    for _ in range(30):
        E = E - (E - e * np.sin(E) - mean_anom) / (1.0 - e * np.cos(E))
    cos_e, sin_e = np.cos(E), np.sin(E)
    b = a * np.sqrt(1.0 - e * e)
    x_orb, y_orb = a * (cos_e - e), b * sin_e
    n_mean = np.sqrt(mu / a ** 3)
    rdot = n_mean * a / (1.0 - e * cos_e)
    vx_orb, vy_orb = -a * sin_e * rdot / a, b * cos_e * rdot / a
    co, so = np.cos(node), np.sin(node)
    cw, sw = np.cos(peri), np.sin(peri)
    ci, si = np.cos(inc), np.sin(inc)
    r11, r12 = co * cw - so * sw * ci, -co * sw - so * cw * ci
    r21, r22 = so * cw + co * sw * ci, -so * sw + co * cw * ci
    r31, r32 = sw * si, cw * si
    pos = (r11 * x_orb + r12 * y_orb, r21 * x_orb + r22 * y_orb, r31 * x_orb + r32 * y_orb)
    vel = (r11 * vx_orb + r12 * vy_orb, r21 * vx_orb + r22 * vy_orb, r31 * vx_orb + r32 * vy_orb)
    return pos, vel


def collisional_disk(n: int = 262144, seed: int = 2, radius_scale: float = 1000.0,
                     central_mass: float = 1.0) -> Bodies:
    """Keplerian disk around a central mass (body 0) plus n bodies: semi-major
    axes U[0.5, 5] AU, log-uniform masses [1e-9, 1e-6] Msun, eccentricities and
    inclinations Rayleigh(0.01), radii from a 3 g/cm^3 density scaled by
    `radius_scale`.  Densities are set consistently with the scaled radii so
    the density-preserving merge (collision_resolver.cpp:205-216) keeps them."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.uniform(0.5, 5.0, n)
    e = np.minimum(rng.rayleigh(0.01, n), 0.9)
    inc = rng.rayleigh(0.01, n)
    node, peri, manom = (2.0 * np.pi * rng.random(n) for _ in range(3))
    m = 10.0 ** rng.uniform(-9.0, -6.0, n)
    (x, y, z), (vx, vy, vz) = _kepler_state(a, e, inc, node, peri, manom, central_mass)
    rad = radius_scale * np.cbrt(3.0 * m / (4.0 * np.pi * DENSITY_3GCC_MSUN_AU3))
    dens = m / ((4.0 / 3.0) * np.pi * rad ** 3)
    sun_r = 0.00465047
    cat = lambda c, v: np.concatenate([[c], v])  # noqa: E731
    return Bodies(px=cat(0.0, x), py=cat(0.0, y), pz=cat(0.0, z), vx=cat(0.0, vx),
                  vy=cat(0.0, vy), vz=cat(0.0, vz), mass=cat(central_mass, m),
                  radius=cat(sun_r, rad),
                  density=cat(central_mass / ((4.0 / 3.0) * np.pi * sun_r ** 3), dens),
                  active=np.ones(n + 1, np.uint8), collidable=np.ones(n + 1, np.uint8))


def ensemble_sizes(systems: int = 512, lo: int = 64, hi: int = 8192, seed: int = 3) -> np.ndarray:
    """System sizes drawn log-uniform in [lo, hi]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), systems))).astype(np.int64)


def ensemble(systems: int = 512, seed: int = 3) -> list[Bodies]:
    """Independent Plummer systems (scale 1 AU, 1 Msun each) of log-uniform size."""
    sizes = ensemble_sizes(systems, seed=seed)
    return [plummer(int(k), 1.0, 1.0, seed=seed * 100003 + s) for s, k in enumerate(sizes)]


def sample_rows(active: np.ndarray, ns: int, seed: int) -> np.ndarray:
    """The bodies nb_force_error samples: the first `ns` entries of a
    SplitMix64-driven partial Fisher-Yates shuffle of the active rows in
    index order (all active rows when ns <= 0 or ns >= their count).  The
    shuffle is kept sparse (only displaced positions are stored), so a few
    thousand draws from millions of rows cost milliseconds."""
    cand = np.flatnonzero(np.asarray(active) != 0)
    na = len(cand)
    if ns <= 0 or ns >= na:
        return cand.copy()
    mask = (1 << 64) - 1
    x = int(seed) & mask
    moved: dict[int, int] = {}
    out = np.empty(ns, np.int64)
    for k in range(ns):
        x = (x + 0x9E3779B97F4A7C15) & mask
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        j = k + z % (na - k)
        vk, vj = moved.get(k, k), moved.get(j, j)
        moved[k], moved[j] = vj, vk
        out[k] = cand[vj]
    return out
