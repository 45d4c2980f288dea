"""Seeded synthetic Mg-H systems with the shapes of the benchmark workloads.

hcp Mg with lattice constant ``a`` and ``c = c_over_a * a``; Mg basis
(0,0,0), (1/3,2/3,1/2) of the hexagonal cell; tetrahedral interstitial sites
(0,0,3/8), (0,0,5/8), (1/3,2/3,1/8), (1/3,2/3,7/8).  Species are atomic
numbers (H = 1, Mg = 12), the encoding of the reference's AtomicSpecie enum
(src/Macros.hpp:56-175) and of its dump files (src/IO/dump-input.cpp:193-198).

Every generator returns a dict with
  q        (N, 3) float64 mean positions
  sigma    (N,)   float64 Gaussian widths
  x        (N,)   float64 occupancies
  species  (N,)   int32
  beta, gamma (N,) float64 thermal / chemical multipliers
  origin   (3,)   box origin
  cell     (3, 3) lattice vectors as rows (zero rows for open axes)
  periodic (3,)   int32 flags
"""
from __future__ import annotations

import numpy as np

K_B = 8.617332478e-5  # eV/K (reference src/Macros.hpp:849)
H, MG = 1, 12
A_MG = 3.209
C_OVER_A = 1.624

_MG_BASIS = np.array([[0.0, 0.0, 0.0], [1.0 / 3.0, 2.0 / 3.0, 0.5]])
_TET_BASIS = np.array([[0.0, 0.0, 3.0 / 8.0], [0.0, 0.0, 5.0 / 8.0],
                       [1.0 / 3.0, 2.0 / 3.0, 1.0 / 8.0],
                       [1.0 / 3.0, 2.0 / 3.0, 7.0 / 8.0]])


def hex_vectors(a=A_MG, c_over_a=C_OVER_A):
    c = a * c_over_a
    return np.array([[a, 0.0, 0.0], [-0.5 * a, 0.5 * np.sqrt(3.0) * a, 0.0],
                     [0.0, 0.0, c]])


def ortho_vectors(a=A_MG, c_over_a=C_OVER_A):
    return np.array([[a, 0.0, 0.0], [0.0, np.sqrt(3.0) * a, 0.0],
                     [0.0, 0.0, a * c_over_a]])


# Ortho-hexagonal 4-atom cell a x sqrt(3)a x c; tetrahedral sites follow from
# the hexagonal ones by the same change of basis.
_ORTHO_MG = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0],
                      [0.0, 1.0 / 3.0, 0.5], [0.5, 5.0 / 6.0, 0.5]])


def _ortho_tet():
    out = []
    for sh in ([0.0, 0.0, 0.0], [0.5, 0.5, 0.0]):
        for t in _TET_BASIS:
            # hexagonal fractional (f1, f2, f3) -> cartesian -> ortho fractional
            hv = hex_vectors(1.0, 1.0)
            r = t @ hv
            f = np.array([r[0], r[1] / np.sqrt(3.0), t[2]]) + sh
            out.append(f % 1.0)
    return np.array(out)


_ORTHO_TET = _ortho_tet()


def _fill(n, rng, kind_sigma, kind_x):
    return kind_sigma(rng, n), kind_x(rng, n)


def _finish(q, species, sigma, x, T, origin, cell, periodic, gamma=0.0):
    n = len(q)
    beta = np.full(n, 1.0 / (K_B * T))
    return dict(q=np.ascontiguousarray(q, dtype=np.float64),
                sigma=np.ascontiguousarray(sigma, dtype=np.float64),
                x=np.ascontiguousarray(x, dtype=np.float64),
                species=np.ascontiguousarray(species, dtype=np.int32),
                beta=beta, gamma=np.full(n, float(gamma)),
                origin=np.asarray(origin, dtype=np.float64),
                cell=np.asarray(cell, dtype=np.float64),
                periodic=np.asarray(periodic, dtype=np.int32))


def supercell(nx, ny, nz, *, ortho=False, a=A_MG, c_over_a=C_OVER_A,
              h_fraction=1.0, x_range=(1.0, 1.0), sigma_range=(0.1, 0.1),
              jitter=0.0, T=300.0, seed=0, with_tetra=True):
    """Periodic hcp Mg(-H) supercell.

    ortho=False: nx*ny*nz hexagonal 2-atom cells (triclinic box).
    ortho=True:  nx*ny*nz ortho-hexagonal 4-atom cells (orthogonal box).
    A seeded fraction ``h_fraction`` of the tetrahedral sites carries H with
    occupancy x ~ U[x_range]; Mg has x = 1.  sigma ~ U[sigma_range] for all
    sites; positions get N(0, jitter) noise.  Sites are ordered Mg first, then
    H, each in cell order.
    """
    rng = np.random.default_rng(seed)
    vec = ortho_vectors(a, c_over_a) if ortho else hex_vectors(a, c_over_a)
    mg_b = _ORTHO_MG if ortho else _MG_BASIS
    tet_b = _ORTHO_TET if ortho else _TET_BASIS
    cells = np.array([[i, j, k] for k in range(nz) for j in range(ny)
                      for i in range(nx)], dtype=np.float64)
    mg_f = (cells[:, None, :] + mg_b[None, :, :]).reshape(-1, 3)
    q_mg = mg_f @ vec
    qs = [q_mg]
    sp = [np.full(len(q_mg), MG, np.int32)]
    xs = [np.ones(len(q_mg))]
    if with_tetra:
        tet_f = (cells[:, None, :] + tet_b[None, :, :]).reshape(-1, 3)
        keep = rng.random(len(tet_f)) < h_fraction if h_fraction < 1.0 else \
            np.ones(len(tet_f), bool)
        q_h = tet_f[keep] @ vec
        qs.append(q_h)
        sp.append(np.full(len(q_h), H, np.int32))
        xs.append(rng.uniform(x_range[0], x_range[1], len(q_h)))
    q = np.concatenate(qs)
    species = np.concatenate(sp)
    x = np.concatenate(xs)
    sigma = rng.uniform(sigma_range[0], sigma_range[1], len(q))
    if jitter > 0:
        q = q + rng.normal(0.0, jitter, q.shape)
    cell = vec * np.array([nx, ny, nz])[:, None]
    # wrap into the cell (fractional in [0,1))
    frac = q @ np.linalg.inv(cell)
    frac -= np.floor(frac)
    q = frac @ cell
    return _finish(q, species, sigma, x, T, np.zeros(3), cell, [1, 1, 1])


def cluster(shape, R, *, length=None, a=A_MG, c_over_a=C_OVER_A,
            x_fn=None, sigma_range=(0.1, 0.1), T=300.0, seed=0,
            h_fraction=1.0):
    """hcp sphere (shape='sphere', radius R) or nanowire along c
    (shape='wire', radius R, ``length`` hexagonal cells, periodic along z).
    ``x_fn(rng, r_xy, n)`` gives H occupancies from the distance to the axis
    (wire) or centre (sphere)."""
    rng = np.random.default_rng(seed)
    vec = hex_vectors(a, c_over_a)
    c = a * c_over_a
    n_ab = int(np.ceil(R / a)) + 2
    nz = length if shape == "wire" else int(np.ceil(R / c)) + 2
    ks = range(nz) if shape == "wire" else range(-nz, nz + 1)
    cells = np.array([[i, j, k] for k in ks for j in range(-2 * n_ab, 2 * n_ab + 1)
                      for i in range(-2 * n_ab, 2 * n_ab + 1)], dtype=np.float64)

    def pick(basis):
        f = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)
        p = f @ vec
        if shape == "wire":
            r = np.hypot(p[:, 0], p[:, 1])
        else:
            r = np.linalg.norm(p, axis=1)
        m = r <= R
        return p[m], r[m]

    q_mg, _ = pick(_MG_BASIS)
    q_h, r_h = pick(_TET_BASIS)
    if h_fraction < 1.0:
        keep = rng.random(len(q_h)) < h_fraction
        q_h, r_h = q_h[keep], r_h[keep]
    x_h = x_fn(rng, r_h, len(q_h)) if x_fn else np.ones(len(q_h))
    q = np.concatenate([q_mg, q_h])
    species = np.concatenate([np.full(len(q_mg), MG, np.int32),
                              np.full(len(q_h), H, np.int32)])
    x = np.concatenate([np.ones(len(q_mg)), x_h])
    sigma = rng.uniform(sigma_range[0], sigma_range[1], len(q))
    if shape == "wire":
        Lz = length * c
        q[:, 2] = np.mod(q[:, 2], Lz)
        lo = q.min(axis=0) - 1.0
        cell = np.zeros((3, 3))
        cell[0, 0] = q[:, 0].max() + 1.0 - lo[0]
        cell[1, 1] = q[:, 1].max() + 1.0 - lo[1]
        cell[2, 2] = Lz
        origin = np.array([lo[0], lo[1], 0.0])
        periodic = [0, 0, 1]
    else:
        lo = q.min(axis=0) - 1.0
        cell = np.diag(q.max(axis=0) + 1.0 - lo)
        origin = lo
        periodic = [0, 0, 0]
    return _finish(q, species, sigma, x, T, origin, cell, periodic)


def config1(seed=1):
    """Periodic hcp Mg 5x5x5 hexagonal cells (250 Mg), H on a seeded 20% of
    the tetrahedral sites with x ~ U[0, 0.1], sigma = 0.1, T = 300 K."""
    return supercell(5, 5, 5, h_fraction=0.2, x_range=(0.0, 0.1),
                     sigma_range=(0.1, 0.1), T=300.0, seed=seed)


def config2(seed=2):
    """Periodic hcp Mg 20x15x15 hexagonal cells (9000 Mg + 18000 tetrahedral
    H sites, x ~ U[0, 0.3]), jitter N(0, 0.02), sigma ~ U[0.08, 0.15], 400 K."""
    return supercell(20, 15, 15, h_fraction=1.0, x_range=(0.0, 0.3),
                     sigma_range=(0.08, 0.15), jitter=0.02, T=400.0, seed=seed)


def config3(seed=3):
    """hcp Mg nanowire, radius 30 A along c, 20 cells long, periodic along the
    axis; H x ~ U[0, 0.5] for r > 20 A and 0.02 inside."""
    def xf(rng, r, n):
        x = np.full(n, 0.02)
        m = r > 20.0
        x[m] = rng.uniform(0.0, 0.5, m.sum())
        return x
    return cluster("wire", 30.0, length=20, x_fn=xf, seed=seed)


def sphere(R, *, T=300.0, h_fraction=0.5, seed=0):
    """hcp Mg-H sphere of radius R with H on a seeded fraction of sites."""
    def xf(rng, r, n):
        return rng.uniform(0.0, 0.5, n)
    return cluster("sphere", R, x_fn=xf, T=T, h_fraction=h_fraction, seed=seed)


def config4(n=128, seed=4):
    """n independent spheres, radii log-uniform on [8, 25] A, per-sphere
    T ~ U[300, 600] K and H fraction ~ U[0, 0.5]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        R = float(np.exp(rng.uniform(np.log(8.0), np.log(25.0))))
        T = float(rng.uniform(300.0, 600.0))
        hf = float(rng.uniform(0.0, 0.5))
        out.append(sphere(R, T=T, h_fraction=hf, seed=seed * 1000 + k))
    return out


def periodic_cube(n_mg, *, h_fraction=0.3, T=300.0, seed=0):
    """Periodic ortho-hexagonal block of about n_mg Mg (4 per cell), as close
    to a cube as whole cells allow and at least 2 rc thick along every axis,
    H on a seeded fraction of the tetrahedral sites with x ~ U[0, 0.3]."""
    dims = np.array([A_MG, np.sqrt(3.0) * A_MG, C_OVER_A * A_MG])
    edge = (n_mg / 4.0 * np.prod(dims)) ** (1.0 / 3.0)
    n = np.maximum(np.round(edge / dims).astype(int), [4, 3, 3])
    return supercell(int(n[0]), int(n[1]), int(n[2]), ortho=True, h_fraction=h_fraction,
                     x_range=(0.0, 0.3), sigma_range=(0.08, 0.15), jitter=0.02, T=T,
                     seed=seed)


def wire(R, length, *, T=300.0, seed=0):
    """hcp nanowire of radius R along c, ``length`` cells, periodic along the
    axis; H x ~ U[0, 0.5] beyond 2/3 R and 0.02 inside (the precision
    workload's profile, scaled)."""
    def xf(rng, r, n):
        x = np.full(n, 0.02)
        m = r > (2.0 / 3.0) * R
        x[m] = rng.uniform(0.0, 0.5, m.sum())
        return x
    return cluster("wire", R, length=length, x_fn=xf, T=T, seed=seed)


def config5(n_jobs=64, rate=200.0, seed=5):
    """The served job stream: Poisson arrivals (mean ``rate`` jobs/s) of
    relaxation and 100-step master-equation jobs, half and half, on periodic
    cubes of 250-60 000 Mg (log-uniform), nanowires (R ~ U[10, 30] A, 4-20
    cells) and spheres (R log-uniform on [8, 25] A), T ~ U[300, 600] K.
    Returns a list of (arrival time [s], system, job kind)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    jobs = []
    for k in range(n_jobs):
        T = float(rng.uniform(300.0, 600.0))
        shape = rng.choice(["cube", "cube", "wire", "sphere"])
        s_seed = seed * 100000 + k
        if shape == "cube":
            n_mg = float(np.exp(rng.uniform(np.log(250.0), np.log(60000.0))))
            s = periodic_cube(n_mg, h_fraction=float(rng.uniform(0.0, 0.5)), T=T, seed=s_seed)
        elif shape == "wire":
            s = wire(float(rng.uniform(10.0, 30.0)), int(rng.integers(4, 21)), T=T, seed=s_seed)
        else:
            R = float(np.exp(rng.uniform(np.log(8.0), np.log(25.0))))
            s = sphere(R, T=T, h_fraction=float(rng.uniform(0.0, 0.5)), seed=s_seed)
        kind = "relax" if rng.random() < 0.5 else "dmd"
        jobs.append((float(t[k]), s, kind))
    return jobs
