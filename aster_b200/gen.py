"""Seeded synthetic initial conditions for the force/integration hot path.

The reference only ships unseeded ``std::rand`` disks and noise "cosmic webs"
(src/clusters/presets_impl.cpp:70-296); none of the distributions below exist
there. Each generator restates a published sampling method, is fully
determined by its integer seed (numpy PCG64), and returns FP64 arrays:
positions (n,3), velocities (n,3), masses (n,).

Units: G = 1 unless stated. All systems are centred to zero centre-of-mass
position and velocity unless stated.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "plummer",
    "exponential_disk",
    "hierarchical_ensemble",
    "planetary_system",
    "lognormal_masses",
    "com_centre",
    "bounding_cube",
]


def com_centre(pos: np.ndarray, vel: np.ndarray, m: np.ndarray):
    """Shift to zero centre-of-mass position and velocity (in place copies)."""
    M = m.sum()
    pos = pos - (m[:, None] * pos).sum(0) / M
    vel = vel - (m[:, None] * vel).sum(0) / M
    return pos, vel


def bounding_cube(pos: np.ndarray) -> float:
    """Half-width B of the origin-centred cube holding every body:
    B = max_i max(|x_i|, |y_i|, |z_i|). Morton codes normalise by it."""
    return float(np.abs(pos).max())


def lognormal_masses(n: int, rng: np.random.Generator, mu: float, sigma: float,
                     total: float | None = 1.0) -> np.ndarray:
    m = rng.lognormal(mean=mu, sigma=sigma, size=n)
    if total is not None:
        m *= total / m.sum()
    return m


def _isotropic(n: int, rng: np.random.Generator) -> np.ndarray:
    cos_t = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    sin_t = np.sqrt(1.0 - cos_t * cos_t)
    return np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t], axis=1)


def plummer(n: int, seed: int, a: float = 1.0, M: float = 1.0, G: float = 1.0,
            r_cut: float = 10.0, masses: str = "equal", mass_sigma: float = 0.5):
    """Plummer sphere by the Aarseth, Henon & Wielen (1974) method.

    Radius: r = a / sqrt(X^(-2/3) - 1), X ~ U(0,1], rejecting r > r_cut * a
    (stated radial cut; 98.5% of the mass lies inside 10a). Speed: q = v/v_esc
    sampled by von Neumann rejection on g(q) = q^2 (1-q^2)^(7/2) (bound 0.1),
    v_esc = sqrt(2 G M / a) (1 + r^2/a^2)^(-1/4); isotropic directions.
    masses: "equal" (M/n each) or "lognormal" (mu=0, sigma=mass_sigma,
    renormalised to M). Velocities use the equal-mass distribution function
    in both cases.
    """
    rng = np.random.default_rng(seed)
    r = np.empty(0)
    while r.size < n:
        X = rng.uniform(0.0, 1.0, 2 * (n - r.size) + 16)
        X = X[X > 0]
        rr = a / np.sqrt(X ** (-2.0 / 3.0) - 1.0)
        r = np.concatenate([r, rr[rr <= r_cut * a]])
    r = r[:n]
    pos = _isotropic(n, rng) * r[:, None]
    q = np.empty(0)
    while q.size < n:
        k = 2 * (n - q.size) + 16
        qq = rng.uniform(0.0, 1.0, k)
        yy = rng.uniform(0.0, 0.1, k)
        q = np.concatenate([q, qq[yy < qq * qq * (1.0 - qq * qq) ** 3.5]])
    q = q[:n]
    v_esc = np.sqrt(2.0 * G * M / a) * (1.0 + (r / a) ** 2) ** -0.25
    vel = _isotropic(n, rng) * (q * v_esc)[:, None]
    if masses == "equal":
        m = np.full(n, M / n)
    elif masses == "lognormal":
        m = lognormal_masses(n, rng, 0.0, mass_sigma, total=M)
    else:
        raise ValueError(f"unknown mass spectrum {masses!r}")
    pos, vel = com_centre(pos, vel, m)
    return pos, vel, m


def exponential_disk(n: int, seed: int, Rd: float = 1.0, R_cut: float = 5.0,
                     z0: float = 0.1, M_disk: float = 1.0, M_central: float = 0.1,
                     sigma_frac: float = 0.01, G: float = 1.0):
    """Cold exponential disk plus a central point mass (body 0).

    n counts every body: n-1 disk bodies of mass M_disk/(n-1) and the central
    mass. Surface density exp(-R/Rd) truncated at R_cut*Rd: R ~ Gamma(2, Rd)
    (the radial law of an exponential disk) by rejection. Vertical sech^2(z/z0):
    z = z0 artanh(2U-1). Circular speed from the enclosed mass,
    v_c = sqrt(G (M_central + M_disk(<R)) / R), with M_disk(<R) counted from the
    sampled bodies; tangential velocity plus isotropic Gaussian dispersion of
    sigma_frac * v_c per component.
    """
    rng = np.random.default_rng(seed)
    nd = n - 1
    R = np.empty(0)
    while R.size < nd:
        k = 2 * (nd - R.size) + 16
        rr = rng.gamma(2.0, Rd, k)
        R = np.concatenate([R, rr[rr <= R_cut * Rd]])
    R = R[:nd]
    phi = rng.uniform(0.0, 2.0 * np.pi, nd)
    u = rng.uniform(0.0, 1.0, nd)
    u = np.clip(u, 1e-12, 1.0 - 1e-12)
    z = z0 * np.arctanh(2.0 * u - 1.0)
    md = M_disk / nd
    order = np.argsort(R, kind="stable")
    enclosed = np.empty(nd)
    enclosed[order] = M_central + md * np.arange(nd)
    vc = np.sqrt(G * enclosed / R)
    tang = np.stack([-np.sin(phi), np.cos(phi), np.zeros(nd)], axis=1)
    vel_d = tang * vc[:, None] + rng.normal(0.0, 1.0, (nd, 3)) * (sigma_frac * vc)[:, None]
    pos_d = np.stack([R * np.cos(phi), R * np.sin(phi), z], axis=1)
    pos = np.concatenate([np.zeros((1, 3)), pos_d])
    vel = np.concatenate([np.zeros((1, 3)), vel_d])
    m = np.concatenate([[M_central], np.full(nd, md)])
    pos, vel = com_centre(pos, vel, m)
    return pos, vel, m


def _kepler_E(Mmean: np.ndarray, e: np.ndarray) -> np.ndarray:
    """Eccentric anomaly from mean anomaly (Newton iteration, vectorised)."""
    E = np.where(e < 0.8, Mmean, np.pi * np.ones_like(Mmean))
    for _ in range(60):
        f = E - e * np.sin(E) - Mmean
        E = E - f / (1.0 - e * np.cos(E))
    return E


def hierarchical_ensemble(n_systems: int, seed: int, n_min: int = 3, n_max: int = 64,
                          G: float = 1.0):
    """Few-body hierarchical systems for the batched ensemble.

    Per system: n ~ U{n_min..n_max}; masses lognormal(mu=0, sigma=1) (not
    renormalised); bodies 0,1 form an inner binary with a ~ U[0.01, 0.1],
    e ~ U[0, 0.9], random orientation and uniform mean anomaly; bodies 2..n-1
    sit isotropically at radii ~ U[1, 10] on circular orbits about the mass
    enclosed within their radius, in a random plane. Each system is centred.

    Returns (pos, vel, m, offsets): concatenated FP64 arrays and int64
    offsets[n_systems+1] (system s owns bodies offsets[s]:offsets[s+1]).
    """
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, n_systems)
    offsets = np.zeros(n_systems + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    ntot = int(offsets[-1])
    m = rng.lognormal(0.0, 1.0, ntot)
    pos = np.zeros((ntot, 3))
    vel = np.zeros((ntot, 3))
    i0 = offsets[:-1]
    m0, m1 = m[i0], m[i0 + 1]
    a = rng.uniform(0.01, 0.1, n_systems)
    e = rng.uniform(0.0, 0.9, n_systems)
    Mmean = rng.uniform(0.0, 2.0 * np.pi, n_systems)
    E = _kepler_E(Mmean, e)
    mu = G * (m0 + m1)
    # relative orbit in its own plane
    xr = a * (np.cos(E) - e)
    yr = a * np.sqrt(1.0 - e * e) * np.sin(E)
    n_mean = np.sqrt(mu / a ** 3)
    Edot = n_mean / (1.0 - e * np.cos(E))
    vxr = -a * np.sin(E) * Edot
    vyr = a * np.sqrt(1.0 - e * e) * np.cos(E) * Edot
    # random orientation: orthonormal frame from an isotropic normal
    nrm = _isotropic(n_systems, rng)
    helper = np.where(np.abs(nrm[:, :1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    ex = np.cross(nrm, helper)
    ex /= np.linalg.norm(ex, axis=1, keepdims=True)
    ey = np.cross(nrm, ex)
    rrel = xr[:, None] * ex + yr[:, None] * ey
    vrel = vxr[:, None] * ex + vyr[:, None] * ey
    f0 = (m1 / (m0 + m1))[:, None]
    f1 = (m0 / (m0 + m1))[:, None]
    pos[i0] = -f0 * rrel
    pos[i0 + 1] = f1 * rrel
    vel[i0] = -f0 * vrel
    vel[i0 + 1] = f1 * vrel
    # outer bodies
    sys_of = np.repeat(np.arange(n_systems), sizes)
    local = np.arange(ntot) - offsets[sys_of]
    outer = np.nonzero(local >= 2)[0]
    r_out = rng.uniform(1.0, 10.0, outer.size)
    dirs = _isotropic(outer.size, rng)
    # enclosed mass: binary + outer bodies of the same system at smaller radius
    s_out = sys_of[outer]
    key = np.lexsort((r_out, s_out))
    enc = np.empty(outer.size)
    ms = m[outer][key]
    ss = s_out[key]
    csum = np.cumsum(ms)
    first = np.r_[0, np.nonzero(np.diff(ss))[0] + 1]
    base = np.zeros(outer.size)
    start_idx = np.repeat(first, np.diff(np.r_[first, outer.size]))
    base = csum[start_idx] - ms[start_idx]
    enc_sorted = (csum - ms) - base + (m0 + m1)[ss]
    enc[key] = enc_sorted
    vc = np.sqrt(G * enc / r_out)
    rnd = _isotropic(outer.size, rng)
    t = np.cross(dirs, rnd)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    pos[outer] = dirs * r_out[:, None]
    vel[outer] = t * vc[:, None]
    # centre each system
    Ms = np.add.reduceat(m, i0)
    cp = np.add.reduceat(m[:, None] * pos, i0, axis=0) / Ms[:, None]
    cv = np.add.reduceat(m[:, None] * vel, i0, axis=0) / Ms[:, None]
    pos -= cp[sys_of]
    vel -= cv[sys_of]
    return pos, vel, m, offsets


def planetary_system(n_planets: int, n_particles: int, seed: int, M_star: float = 1.0, G: float = 1.0,
                     planet_mass: tuple = (1e-5, 1e-3), a_range: tuple = (1.0, 30.0),
                     particle_a: tuple = (0.5, 40.0), particle_e: float = 0.6, inclination: float = 0.05):
    """A central star (body 0) with planets and massless test particles.

    Planets: masses log-uniform in planet_mass, semi-major axes log-uniform in
    a_range, e ~ U[0, 0.1]; test particles: m = 0, a log-uniform in particle_a,
    e ~ U[0, particle_e]. All orbits: inclination ~ U[0, inclination] rad,
    uniform node, argument of pericentre and mean anomaly; elements about mu =
    G (M_star + m) (heliocentric), as in Murray & Dermott (1999) ch. 2. The
    system is centred on its barycentre.
    """
    rng = np.random.default_rng(seed)
    n = 1 + n_planets + n_particles
    m = np.zeros(n)
    m[0] = M_star
    m[1:1 + n_planets] = np.exp(rng.uniform(np.log(planet_mass[0]), np.log(planet_mass[1]), n_planets))
    a = np.empty(n - 1)
    e = np.empty(n - 1)
    a[:n_planets] = np.exp(rng.uniform(np.log(a_range[0]), np.log(a_range[1]), n_planets))
    e[:n_planets] = rng.uniform(0.0, 0.1, n_planets)
    a[n_planets:] = np.exp(rng.uniform(np.log(particle_a[0]), np.log(particle_a[1]), n_particles))
    e[n_planets:] = rng.uniform(0.0, particle_e, n_particles)
    inc = rng.uniform(0.0, inclination, n - 1)
    node = rng.uniform(0.0, 2.0 * np.pi, n - 1)
    argp = rng.uniform(0.0, 2.0 * np.pi, n - 1)
    E = _kepler_E(rng.uniform(0.0, 2.0 * np.pi, n - 1), e)
    mu = G * (M_star + m[1:])
    xo = a * (np.cos(E) - e)
    yo = a * np.sqrt(1.0 - e * e) * np.sin(E)
    Edot = np.sqrt(mu / a ** 3) / (1.0 - e * np.cos(E))
    vxo = -a * np.sin(E) * Edot
    vyo = a * np.sqrt(1.0 - e * e) * np.cos(E) * Edot
    cO, sO, cw, sw, ci, si = np.cos(node), np.sin(node), np.cos(argp), np.sin(argp), np.cos(inc), np.sin(inc)
    # perifocal -> reference frame (R_z(node) R_x(inc) R_z(argp))
    px = np.stack([cO * cw - sO * sw * ci, sO * cw + cO * sw * ci, sw * si], axis=1)
    qx = np.stack([-cO * sw - sO * cw * ci, -sO * sw + cO * cw * ci, cw * si], axis=1)
    pos = np.zeros((n, 3))
    vel = np.zeros((n, 3))
    pos[1:] = xo[:, None] * px + yo[:, None] * qx
    vel[1:] = vxo[:, None] * px + vyo[:, None] * qx
    pos, vel = com_centre(pos, vel, m)
    return pos, vel, m


def kepler_orbits(n: int, seed: int, mu: float = 1.0):
    """A unit central mass (body 0, at rest at the origin) and n massless
    bodies on conic orbits about it, for checking Kepler drifts on their own:
    half elliptic (e ~ U[0, 0.95]), a quarter hyperbolic (e ~ U[1.05, 3]) and
    the rest near-parabolic (e ~ U[0.97, 1.03]). Pericentre distance
    log-uniform in [0.3, 5]; true anomaly U[-2, 2] rad, clipped to 0.9 of a
    hyperbola's asymptote angle; each orbit plane turned by a uniform random
    rotation (a normalised Gaussian quaternion). Returns (pos, vel, m, e)."""
    rng = np.random.default_rng(seed)
    e = np.concatenate([rng.uniform(0.0, 0.95, n // 2), rng.uniform(1.05, 3.0, n // 4),
                        rng.uniform(0.97, 1.03, n - n // 2 - n // 4)])
    q = np.exp(rng.uniform(np.log(0.3), np.log(5.0), n))
    f = rng.uniform(-2.0, 2.0, n)
    lim = np.where(e > 1.0, 0.9 * np.arccos(-1.0 / np.maximum(e, 1.0 + 1e-9)), np.pi)
    f = np.clip(f, -lim, lim)
    p = q * (1.0 + e)
    r = p / (1.0 + e * np.cos(f))
    x = np.stack([r * np.cos(f), r * np.sin(f), np.zeros(n)], axis=1)
    v = np.sqrt(mu / p)[:, None] * np.stack([-np.sin(f), e + np.cos(f), np.zeros(n)], axis=1)
    qt = rng.normal(size=(n, 4))
    qt /= np.linalg.norm(qt, axis=1, keepdims=True)
    w, a, b, c = qt.T
    rot = np.stack([np.stack([1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)], 1),
                    np.stack([2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)], 1),
                    np.stack([2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)], 1)], axis=1)
    x = np.einsum("nij,nj->ni", rot, x)
    v = np.einsum("nij,nj->ni", rot, v)
    pos = np.vstack([np.zeros(3), x])
    vel = np.vstack([np.zeros(3), v])
    m = np.zeros(n + 1)
    m[0] = mu
    return pos, vel, m, e


def ensemble_measures(pos, vel, m, offsets, G: float = 1.0):
    """Per system of a hierarchical ensemble (bodies 0, 1 the inner binary):
    the binary's pericentre time sqrt(r_p^3 / (G (m_0 + m_1))), the smallest
    initial separation of any other pair, and the energy scale K + |U|
    (kinetic plus the magnitude of the Newtonian potential energy). Returns
    (t_peri, d_min, scale) as arrays of the system count."""
    off = np.asarray(offsets, dtype=np.int64)
    i0 = off[:-1]
    r, v = pos[i0 + 1] - pos[i0], vel[i0 + 1] - vel[i0]
    mu = G * (m[i0] + m[i0 + 1])
    rn = np.linalg.norm(r, axis=1)
    a = 1.0 / (2.0 / rn - (v * v).sum(1) / mu)
    h = np.cross(r, v)
    e = np.sqrt(np.maximum(0.0, 1.0 - (h * h).sum(1) / (mu * a)))
    tp = np.sqrt((a * (1.0 - e)) ** 3 / mu)
    ns = len(off) - 1
    dmin, scale = np.empty(ns), np.empty(ns)
    for s in range(ns):
        x, u, mm = pos[off[s]:off[s + 1]], vel[off[s]:off[s + 1]], m[off[s]:off[s + 1]]
        d = np.linalg.norm(x[:, None] - x[None], axis=-1)
        iu = np.triu_indices(len(mm), 1)
        pot = G * (mm[:, None] * mm[None] / np.where(d > 0, d, np.inf))[iu].sum()
        scale[s] = 0.5 * (mm * (u * u).sum(1)).sum() + pot
        d[0, 1] = d[1, 0] = np.inf
        np.fill_diagonal(d, np.inf)
        dmin[s] = d.min()
    return tp, dmin, scale
