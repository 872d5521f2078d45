"""Generates the golden vectors in tests/golden/ by running the reference's OWN calc functions
(CalcFunctions.cpp compiled from the reference sources by oracle/Makefile into
oracle/_ref/libxnsref.so) on small seeded synthetic structures.

    make -C oracle REF=<reference source tree> && python tests/golden/make_golden.py [case-prefix ...]

With prefixes, only the cases whose names start with one of them are regenerated (the full-size
cases take about a minute of the reference's CPU code each).

The reference ships no unit tests and no histogram or PDF outputs (its two example patterns need
inputs that cannot be rebuilt here), so these fixtures are the pinned known answers: the CPU test
suite checks the oracle restatement against them and the GPU suite checks the CUDA library against
them.  Each case stores its inputs and the reference's outputs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "softx-d-16-00083_b200"))

from oracle import Reference  # noqa: E402
from xns_b200 import synth  # noqa: E402


def pack(elements):
    return np.concatenate([np.asarray(e).reshape(-1, 3) for e in elements]), np.array([len(e) for e in elements], np.uint32)


def sha256_u64(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def sha256_f64(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def full_size_cases(R, out):
    """The two full-size workloads: the Debye double sum on the 5000-atom fcc sphere (1024 q in
    [0.1, 10), neutron b = 7.63 fm) with its pattern, and the 1.94e5-atom rock-salt cube's histogram at
    0.001 A (30^3 cells, seed 0) as a SHA-256 of its u64 counts (plus its size and total, and the
    hash of the coordinates it was made from, so that a change of the generator shows as such)."""
    sphere = synth.fcc_sphere(n=5000, a=4.078, sigma=0.05, seed=0)
    q = synth.q_mesh(0.1, 10.0, 1024)
    xyz, n = pack(sphere)
    out["debye/fcc5000_neutron"] = dict(xyz=xyz, n_el=n, q=q, source=0, sl=np.array([7.63]), polar=0, lam=0.0,
                                        I=R.int_debye(sphere, q, 0, sl=[7.63]))
    cube = synth.rocksalt_cube(cells=30, a=5.64, vacancy=0.1, sigma=0.07, seed=0)
    nh = R.hist_size(cube, 0.001)
    h = R.hist(cube, nh, 0.001)
    xyz, n = pack(cube)
    out["histhash/rocksalt30_seed0_b0.001"] = dict(n_el=n, bin=0.001, nhist=nh, total=int(h.sum()),
                                                   sha256=sha256_u64(h), xyz_sha256=sha256_f64(xyz))


def main(prefixes=()):
    R = Reference(threads=os.cpu_count() or 4)
    out = {}
    if prefixes:
        full_size_cases(R, out)
        out = {k: v for k, v in out.items() if k.startswith(tuple(prefixes))}
        save(out)
        return

    # 1. histograms: two species rock salt at the reference bin 0.001 and a coarse bin; one-element
    #    fcc sphere; three elements with an empty one and coincident atoms
    rs = synth.rocksalt_cube(cells=3, seed=11)
    sphere = synth.fcc_sphere(n=300, seed=12)
    rng = np.random.default_rng(13)
    tri = [rng.normal(0, 4.0, (70, 3)), np.zeros((0, 3)), rng.normal(0, 4.0, (55, 3))]
    tri[2][5] = tri[0][3]   # a coincident pair across elements
    tri[0][10] = tri[0][2]  # and within an element
    for name, els, bin in (("rocksalt_b0.001", rs, 0.001), ("rocksalt_b0.05", rs, 0.05), ("sphere_b0.001", sphere, 0.001),
                           ("tri_b0.002", tri, 0.002)):
        nh = R.hist_size(els, bin)
        xyz, n = pack(els)
        out["hist/" + name] = dict(xyz=xyz, n_el=n, bin=bin, nhist=nh, hist=R.hist(els, nh, bin),
                                   p0=R.atomic_density(els))

    # 2. Debye double sum: neutron one element, X-ray two elements with polarisation
    q = synth.q_mesh(0.1, 10.0, 128)
    xyz, n = pack(sphere)
    out["debye/sphere_neutron"] = dict(xyz=xyz, n_el=n, q=q, source=0, sl=np.array([7.63]), polar=0, lam=0.0,
                                       I=R.int_debye(sphere, q, 0, sl=[7.63]))
    ff = synth.ff_on_mesh(synth.ff_coefficients(2, seed=14), q)
    xyz, n = pack(rs)
    out["debye/rocksalt_xray_polar"] = dict(xyz=xyz, n_el=n, q=q, source=1, ff=ff, polar=1, lam=1.5,
                                            I=R.int_debye(rs, q, 1, ff=ff, polar=True, lam=1.5))
    qz = synth.q_mesh(0.0, 12.0, 64)  # q = 0 on the mesh
    out["debye/rocksalt_q0"] = dict(xyz=xyz, n_el=n, q=qz, source=0, sl=np.array([3.63, 9.58]), polar=0, lam=0.0,
                                    I=R.int_debye(rs, qz, 0, sl=[3.63, 9.58]))
    # partial Debye: three blocks
    neb = np.array([[30, 20, len(rs[0]) - 50], [25, 25, len(rs[1]) - 50]], dtype=np.uint32)
    out["partial/rocksalt_3blocks"] = dict(xyz=xyz, n_el=n, q=q, source=0, sl=np.array([3.63, 9.58]), n_el_block=neb,
                                           I=R.int_partial_debye(rs, neb, q, 0, sl=[3.63, 9.58]))

    # 3. histogram scenarios: I(q) from the histogram, PDF / RDF / rPDF
    h = out["hist/rocksalt_b0.001"]
    q4 = synth.q_mesh(0.1, 25.0, 256)
    sl = np.array([3.63, 9.58])
    nh4 = R.hist_size(rs, 0.004)  # a coarser bin keeps the floating-point PDF fixtures small
    for pt, pname in ((0, "rdf"), (1, "pdf"), (2, "rpdf")):
        I, pdf = R.pdf_and_debye(rs, nh4, 0.004, 4, pt, h["p0"], q4, 0, sl=sl)
        out["pdf/rocksalt_" + pname] = dict(xyz=h["xyz"], n_el=h["n_el"], bin=0.004, nhist=nh4, p0=h["p0"], q=q4,
                                            sl=sl, pdftype=pt, I=I, pdf=pdf)
    ffq4 = synth.ff_on_mesh(synth.ff_coefficients(2, seed=15), q4)
    out["iqhist/rocksalt_xray"] = dict(hist=h["hist"], n_el=h["n_el"], nhist=h["nhist"], bin=0.001, q=q4, source=1,
                                       ff=ffq4, polar=1, lam=0.9,
                                       I=R.int_1d_hist(h["hist"], h["n_el"], h["nhist"], 0.001, q4, 1, ff=ffq4, polar=True,
                                                       lam=0.9))

    # 4. 2D: polar mesh, X-ray, 2 x 1 x 3 Euler mesh in convention ZYZ
    small = [e[:60] for e in rs]
    q2 = synth.q_mesh(0.5, 8.0, 24)
    ff2 = synth.ff_on_mesh(synth.ff_coefficients(2, seed=16), q2)
    emin, emax, en = np.array([0.0, 0.0, 0.0]), np.array([1.0, 0.5, 2.0]), np.array([2, 1, 3], np.uint32)
    I2D, I = R.int_2d(small, q2, 16, emin, emax, en, 4, 0.7, 1, ff=ff2, polar=True)
    xyz, n = pack(small)
    out["2d/rocksalt_xray"] = dict(xyz=xyz, n_el=n, q=q2, nfi=16, emin=emin, emax=emax, en=en, conv=4, lam=0.7, source=1,
                                   ff=ff2, polar=1, I2D=I2D, I=I)
    I2D, I = R.int_2d(sphere[:1], q2, 20, np.zeros(3), np.zeros(3), np.ones(3, np.uint32), 5, 0.05, 0, sl=[7.63])
    xyz, n = pack(sphere)
    out["2d/sphere_neutron"] = dict(xyz=xyz, n_el=n, q=q2, nfi=20, emin=np.zeros(3), emax=np.zeros(3),
                                    en=np.ones(3, np.uint32), conv=5, lam=0.05, source=0, sl=np.array([7.63]), polar=0,
                                    I2D=I2D, I=I)

    # 5. rotation matrices of all 12 conventions
    eul = np.array([0.3, 1.1, -0.7])
    out["rot/all"] = dict(euler=eul, m=np.stack([R.rot_matrix(eul, c) for c in range(12)]))

    full_size_cases(R, out)
    save(out)


def save(out):
    for key, d in out.items():
        path = os.path.join(HERE, key.replace("/", "__") + ".npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in d.items()})
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main(sys.argv[1:])
