"""Seeded synthetic structures for the benchmark workloads and the parity tests.

Each generator returns a list of per-element (n_e, 3) float64 coordinate arrays (the layout of the
reference's ra[Nel]) plus its scattering weights.  All randomness comes from numpy's PCG64 seeded by
the caller, so a structure is reproducible bit for bit.

Workloads (sizes as stated, reduced sizes for tests):
  fcc_sphere     fcc lattice cropped to the n atoms nearest the centre, Gaussian displacement per axis
                 (Debye double sum: a = 4.078 A, 5000 atoms, sigma 0.05 A, b = 7.63 fm)
  rocksalt_cube  two-species rock salt nanocube with vacancies and Gaussian displacement
                 (histogram + I(q) + PDF: a = 5.64 A, 30^3 cells ~ 1.94e5 atoms, 10 % vacancies,
                 sigma 0.07 A, b = 3.63 / 9.58 fm)
  fcc_crystallite fcc cube with random substitution by a second species, rotated by a seeded
                 quaternion (2D amplitude: a = 3.61 A, ~1e6 atoms, 5 % substitution)
  atom_file_block a structure read from an atom list (one cell, no symmetry) as a builder block: sites
                 at random in a cube of the given density, a fraction planted within N(0, 0.1 A) of
                 earlier sites, partial occupancy on every third site (structure builder: 2e5 sites)
  rocksalt_block the rock-salt cube as the reference's XML describes it: a two-site cell with the four
                 fcc translations, replicated, with occupancy and displacement per site
"""
import numpy as np


def _fcc_cells(m):
    base = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 1, 3)
    return (g + base[None]).reshape(-1, 3)


def fcc_sphere(n=5000, a=4.078, sigma=0.05, seed=0):
    """The n fcc sites nearest the lattice centre (ties broken by site index), displaced by N(0, sigma)."""
    m = int(np.ceil((n / 4 * 6 / np.pi) ** (1 / 3))) + 3
    sites = _fcc_cells(m) * a
    c = sites.mean(axis=0)
    d2 = ((sites - c) ** 2).sum(axis=1)
    order = np.lexsort((np.arange(len(sites)), np.round(d2, 9)))[:n]
    rng = np.random.default_rng(seed)
    xyz = sites[order] - c + rng.normal(0.0, sigma, size=(n, 3))
    return [xyz]


def sphere_ensemble(count=256, nmin=1000, nmax=200000, a=4.078, smin=0.02, smax=0.1, seed=0):
    """count fcc spheres (one element each) with atom counts log-uniform in [nmin, nmax] and their own
    Gaussian displacement sigma uniform in [smin, smax]: the n sites nearest the lattice centre, as
    fcc_sphere, sorted once for all.  Returns (structures, atom counts, sigmas)."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), count)).astype(np.int64)
    sig = rng.uniform(smin, smax, count)
    m = int(np.ceil((ns.max() / 4 * 6 / np.pi) ** (1 / 3))) + 3
    sites = _fcc_cells(m) * a
    c = sites.mean(axis=0)
    d2 = ((sites - c) ** 2).sum(axis=1)
    order = np.lexsort((np.arange(len(sites)), np.round(d2, 9)))[:ns.max()]
    base = sites[order] - c
    structs = [[base[:n] + rng.normal(0.0, s, size=(n, 3))] for n, s in zip(ns, sig)]
    return structs, ns, sig


def rocksalt_cube(cells=30, a=5.64, vacancy=0.1, sigma=0.07, seed=0):
    """Rock-salt cube of cells^3 unit cells; species 0 (Na) on the fcc sites, species 1 (Cl) on the
    half-shifted ones.  Returns [na, cl]."""
    na = _fcc_cells(cells) * a
    cl = na + np.array([0.5, 0.0, 0.0]) * a
    rng = np.random.default_rng(seed)
    out = []
    for s in (na, cl):
        keep = rng.random(len(s)) >= vacancy
        s = s[keep]
        out.append(s + rng.normal(0.0, sigma, size=s.shape))
    c = np.concatenate(out).mean(axis=0)
    return [o - c for o in out]


def _quat_matrix(qt):
    w, x, y, z = qt / np.linalg.norm(qt)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def fcc_crystallite(cells=63, a=3.61, subst=0.05, seed=0):
    """fcc cube of cells^3 unit cells (4 cells^3 atoms), a fraction subst of sites replaced by a second
    species, rotated by a seeded random quaternion about the centre.  Returns [host, substituent]."""
    rng = np.random.default_rng(seed)
    sites = _fcc_cells(cells) * a
    sites -= sites.mean(axis=0)
    sites = sites @ _quat_matrix(rng.normal(size=4)).T
    sub = rng.random(len(sites)) < subst
    return [sites[~sub], sites[sub]]


def random_cluster(n, density=0.085, seed=0):
    """Random close packing stand-in: n points uniform in a sphere of the given density."""
    rng = np.random.default_rng(seed)
    R = (3 * n / (4 * np.pi * density)) ** (1 / 3)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return [v * R * rng.random(n)[:, None] ** (1 / 3)]


def ff_coefficients(nel, seed=0):
    """Seeded X-ray form-factor coefficients a_k in [0.5, 12], b_k in [0.1, 60], c in [0, 2] (k = 1..4)
    for f(q) = sum_k a_k exp(-b_k (q/4pi)^2) + c; returns (nel, 9) [a1..a4, b1..b4, c]."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.5, 12, size=(nel, 4))
    b = rng.uniform(0.1, 60, size=(nel, 4))
    c = rng.uniform(0, 2, size=(nel, 1))
    return np.concatenate([a, b, c], axis=1)


def ff_on_mesh(coef, q):
    """Form factors of ff_coefficients rows on a q mesh: (nel, nq)."""
    s2 = (np.asarray(q) / (4 * np.pi)) ** 2
    return np.stack([(c[:4, None] * np.exp(-c[4:8, None] * s2[None])).sum(0) + c[8] for c in coef])


def q_mesh(qmin, qmax, n):
    """The reference's q mesh: q[i] = qmin + i*(qmax-qmin)/n, qmax excluded (ReadXML.cpp:220-222)."""
    dq = (qmax - qmin) / n
    return np.array([qmin + i * dq for i in range(n)], dtype=np.float64)


def hist_size(elements, bin):
    """GetHistSize (CalcFunctions.cpp:224-243): (unsigned)(|bbox diagonal| / bin) + 1."""
    xyz = np.concatenate([np.asarray(e).reshape(-1, 3) for e in elements])
    d = xyz.max(axis=0) - xyz.min(axis=0)
    return int(np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / bin) + 1


def atom_file_block(n=200000, density=0.05, planted=0.02, occ=0.6, seed=1):
    """A builder block for an atom list of n sites (two elements, halves), see the module docstring."""
    from .structure import Block
    rng = np.random.default_rng(seed)
    pts = rng.uniform(0, (n / density) ** (1 / 3), (n, 3))
    k = int(n * planted)
    pts[n // 2:n // 2 + k] = pts[:k] + rng.normal(0, 0.1, (k, 3))
    return Block(pts, [n // 2, n - n // 2], [0, 1], occ=np.where(np.arange(n) % 3 == 0, occ, 1.0))


def rocksalt_block(cells=30, a=5.64, vacancy=0.1, sigma=0.07):
    """The rock-salt cube as a builder block (Na at 0 0 0, Cl at 1/2 0 0, fcc translations)."""
    from .structure import Block
    fcc = [(np.eye(3), t) for t in [(0, 0, 0), (0, .5, .5), (.5, 0, .5), (.5, .5, 0)]]
    return Block.crystal(np.eye(3) * a, [(0, 0, 0), (0.5, 0, 0)], [1, 1], [0, 1], (cells, cells, cells), symm=fcc,
                         occ=[1 - vacancy] * 2, dev=[sigma] * 2)
