"""CPU: the oracle's restatement of block::calcAtoms (CalcFunctions.cpp:251-392) pinned against the
reference's own calcAtoms compiled from its sources.

Draw-free inputs (full or zero occupancies, no displacements, no molecule rotation) give the same
atoms in the same order bit for bit.  With random draws the reference seeds from the clock, so the
oracle (Philox draws) and the reference are compared by distribution: occupancy fractions and the
displacement vectors' radii and directions."""
import os

import numpy as np
import pytest

from oracle import REF_SO, Oracle, Reference
from xns_b200.structure import Block

needs_reference = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
_LIBS = {}


def oracle():
    if "o" not in _LIBS:
        _LIBS["o"] = Oracle()
    return _LIBS["o"]


def reference():
    if "r" not in _LIBS:
        _LIBS["r"] = Reference()
    return _LIBS["r"]

A_NACL = 5.64
FCC = [(np.eye(3), t) for t in [(0, 0, 0), (0, .5, .5), (.5, 0, .5), (.5, .5, 0)]]


def rocksalt(ncell, occ=None, dev=None, **kw):
    return Block.crystal(np.eye(3) * A_NACL, [(0, 0, 0), (0.5, 0, 0)], [1, 1], [0, 1], ncell, symm=FCC, occ=occ, dev=dev,
                         **kw)


def rot(a, b, c):
    """a rotation matrix from three angles (any orthogonal matrix will do here)"""
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    rz = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rx = np.array([[1, 0, 0], [0, cc, -sc], [0, sc, cc]])
    return rz @ ry @ rx


def same(xa, xb):
    return len(xa) == len(xb) and all(np.array_equal(p, q) for p, q in zip(xa, xb))


def test_philox_known_answers():
    """Philox4x32-10 against the known-answer vectors published with the Random123 library."""
    o = oracle()
    assert list(o.philox([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(o.philox([0xffffffff] * 4, [0xffffffff] * 2)) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(o.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0])) == [
        0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def draw_free_cases():
    """Blocks whose build does not depend on any random draw."""
    cases = {}
    cases["rocksalt_3"] = ([rocksalt((3, 3, 3))], 2)
    # triclinic cell, three elements, symmetry with a rotation part, 2 x 3 x 4 cells
    e = np.array([[4.1, 0.0, 0.0], [0.9, 3.7, 0.0], [0.4, 0.6, 5.2]])
    inv = [(np.eye(3), (0, 0, 0)), (-np.eye(3), (0.5, 0.5, 0.5))]
    cases["triclinic_inversion"] = ([Block.crystal(e, [(0.1, 0.2, 0.3), (0.25, 0.25, 0.25), (0.6, 0.1, 0.9),
                                                     (0.7, 0.45, 0.15)], [2, 1, 1], [0, 1, 2], (2, 3, 4), symm=inv)], 3)
    # sites on a symmetry element: inversion through the origin maps (0,0,0) onto itself, so the
    # second copy merges with the first; (0.999, 0, 0) meets (0.001, 0, 0) across a cell boundary
    cases["merged_sites"] = ([Block.crystal(np.eye(3) * 3.0, [(0, 0, 0), (0.999, 0, 0), (0.001, 0, 0), (0.5, 0.5, 0.5)],
                                            [2, 2], [0, 1], (3, 2, 2), symm=[(np.eye(3), (0, 0, 0)), (-np.eye(3), (0, 0, 0))],
                                            occ=[1.0, 1.0, 1.0, 1.0])], 2)
    # running occupancy: element 0 with occupancy 0 then element 1 with occupancy 1 on one site -> always
    # element 1; two element-0 sites of occupancies 0 and 1 on one site -> the sum stays 0: no atom
    cases["occupancy_rule"] = ([Block(np.array([[0, 0, 0], [1.0, 1.0, 1.0], [0.1, 0, 0], [1.1, 1.0, 1.0]]), [2, 2], [0, 1],
                                      occ=[0.0, 0.0, 1.0, 1.0], e=np.eye(3) * 2.5, ncell=(2, 2, 2))], 2)
    cases["occupancy_rule_same_element"] = ([Block(np.array([[0, 0, 0], [0.1, 0, 0], [1.0, 1.0, 1.0]]), [3], [0],
                                                   occ=[0.0, 1.0, 1.0], e=np.eye(3) * 2.5, ncell=(1, 1, 1))], 1)
    # copies with rotations, a spherical cut-off and a cut-off on the copies; two blocks
    b1 = rocksalt((4, 4, 4), centered=True, r_copy=[(0, 0, 0), (30.0, 1.0, -2.0), (-5.0, 40.0, 3.0)],
                  cf=[np.eye(3), rot(0.3, 0.2, 0.1), rot(-1.0, 0.5, 2.0)], rcut=9.0, rcut_copies=25.0)
    b2 = Block(np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.54]]), [2], [2], e=np.eye(3) * 4.0, ncell=(2, 1, 3),
               r_copy=[(1.0, 2.0, 3.0)], cf=[rot(0.7, -0.4, 1.1)])
    cases["copies_cutoffs_two_blocks"] = ([b1, b2], 3)
    # an atom-file block: one cell, no symmetry, some sites within 0.5 A of each other
    rng = np.random.default_rng(5)
    pts = rng.uniform(0, 30, (3000, 3))
    pts[1500:1600] = pts[:100] + rng.normal(0, 0.1, (100, 3))
    cases["atom_file"] = ([Block(pts, [2000, 1000], [1, 0], occ=np.ones(3000))], 2)
    # every site vacant (occupancy 0: a draw of exactly 0 is the only way in, probability 2^-53)
    cases["all_vacant"] = ([rocksalt((3, 3, 3), occ=[0.0, 0.0])], 2)
    return cases


@needs_reference
@pytest.mark.parametrize("name", sorted(draw_free_cases()))
def test_draw_free_builds_match_reference(name):
    blocks, nel = draw_free_cases()[name]
    xo, nao = oracle().build_atoms(blocks, nel, seed=11)
    xr, nar = reference().calc_atoms(blocks, nel)
    assert [len(x) for x in xo] == [len(x) for x in xr]
    assert np.array_equal(nao, nar)
    assert same(xo, xr)


@needs_reference
def test_merge_cases_are_not_trivial():
    """the draw-free cases exercise the merge: fewer atoms than sites x cells"""
    blocks, nel = draw_free_cases()["merged_sites"]
    xr, _ = reference().calc_atoms(blocks, nel)
    assert sum(len(x) for x in xr) < 4 * 2 * 12
    blocks, nel = draw_free_cases()["occupancy_rule"]
    xr, _ = reference().calc_atoms(blocks, nel)
    assert len(xr[0]) == 0 and len(xr[1]) == 8 * 2
    blocks, nel = draw_free_cases()["occupancy_rule_same_element"]
    xr, _ = reference().calc_atoms(blocks, nel)
    assert len(xr[0]) == 1
    blocks, nel = draw_free_cases()["atom_file"]
    xr, _ = reference().calc_atoms(blocks, nel)
    assert 2700 < sum(len(x) for x in xr) < 2950  # ~100 planted and ~90 chance close pairs


def test_seed_reproducible_and_different():
    b = rocksalt((5, 5, 5), occ=[0.9, 0.9], dev=[0.05, 0.05])
    x1, _ = oracle().build_atoms([b], 2, seed=3)
    x2, _ = oracle().build_atoms([b], 2, seed=3)
    x3, _ = oracle().build_atoms([b], 2, seed=4)
    assert same(x1, x2)
    assert not same(x1, x3)


@needs_reference
def test_vacancies_match_reference_statistically():
    """10 % vacant sites: the fraction of placed atoms agrees within 6 binomial sigmas"""
    b = rocksalt((10, 10, 10), occ=[0.9, 0.9])
    n = 8000
    for xs in (oracle().build_atoms([b], 2, seed=7)[0], reference().calc_atoms([b], 2)[0]):
        for x in xs:
            assert abs(len(x) - 0.9 * n / 2) < 6 * np.sqrt(n / 2 * 0.09)


@needs_reference
def test_shared_site_fractions_match_reference():
    """one site shared by element 0 (occupancy 0.3) and element 1 (0.7): always one atom, 30 % element 0"""
    b = Block(np.array([[0, 0, 0], [0, 0, 0]]), [1, 1], [0, 1], occ=[0.3, 0.7], e=np.eye(3) * 3.0, ncell=(20, 20, 20))
    for xs in (oracle().build_atoms([b], 2, seed=8)[0], reference().calc_atoms([b], 2)[0]):
        assert len(xs[0]) + len(xs[1]) == 8000
        assert abs(len(xs[0]) - 2400) < 6 * np.sqrt(8000 * 0.21)


def _displacements(xs, ideal):
    return np.concatenate([x - i for x, i in zip(xs, ideal)])


@needs_reference
def test_displacements_match_reference_in_distribution():
    """per-atom displacement: radius |N(0, dev)| and direction theta = pi U, phi = 2 pi U (not uniform on
    the sphere); Kolmogorov-Smirnov between the reference's and the oracle's vectors"""
    from scipy.stats import ks_2samp
    dev = 0.07
    ideal, _ = reference().calc_atoms([rocksalt((8, 8, 8))], 2)
    b = rocksalt((8, 8, 8), dev=[dev, dev])
    do = _displacements(oracle().build_atoms([b], 2, seed=9)[0], ideal)
    dr = _displacements(reference().calc_atoms([b], 2)[0], ideal)
    for f in (lambda d: np.linalg.norm(d, axis=1), lambda d: d[:, 2] / np.linalg.norm(d, axis=1),
              lambda d: np.arctan2(d[:, 1], d[:, 0])):
        assert ks_2samp(f(do), f(dr)).pvalue > 1e-4
    assert abs(np.linalg.norm(do, axis=1).mean() / (dev * np.sqrt(2 / np.pi)) - 1) < 0.02


@needs_reference
def test_molecule_rotation_and_displacement_match_reference_in_distribution():
    """a two-atom molecule per cell, randomly rotated (ro_mol) and displaced (dev_mol): bond lengths are
    kept, bond directions and the molecule displacement follow the reference's distributions"""
    from scipy.stats import ks_2samp
    b = Block(np.array([[0.3, -0.2, 0.1], [0.3, -0.2, 1.6]]), [1, 1], [0, 1], e=np.eye(3) * 6.0, ncell=(12, 12, 12),
              ro_mol=True, dev_mol=0.1)
    xo = oracle().build_atoms([b], 2, seed=10)[0]
    xr = reference().calc_atoms([b], 2)[0]
    for xs in (xo, xr):
        assert np.allclose(np.linalg.norm(xs[1] - xs[0], axis=1), 1.5, atol=1e-12)
    bo, br = xo[1] - xo[0], xr[1] - xr[0]
    assert ks_2samp(bo[:, 2], br[:, 2]).pvalue > 1e-4
    assert ks_2samp(np.arctan2(bo[:, 1], bo[:, 0]), np.arctan2(br[:, 1], br[:, 0])).pvalue > 1e-4


def random_draw_free_block(seed):
    """A random block whose build draws nothing that matters: occupancies 0 or 1 (a site's draw decides
    nothing then), no displacements, no molecule rotation; triclinic cell, random symmetry operations
    (orthogonal rotations with random translations, so some sites land on others), 1-4 cells per axis
    (up to 125 merge translations), 1-3 copies with random rotations, random cut-offs."""
    rng = np.random.default_rng(seed)
    e = np.diag(rng.uniform(2.5, 6.0, 3)) + np.triu(rng.uniform(-1.0, 1.0, (3, 3)), 1)
    natom = int(rng.integers(1, 7))
    nid = int(rng.integers(1, min(natom, 3) + 1))
    cuts = np.sort(rng.choice(np.arange(1, natom), nid - 1, replace=False)) if nid > 1 else np.array([], int)
    natom_el = np.diff(np.concatenate([[0], cuts, [natom]]))
    ids = rng.choice(4, nid, replace=False)
    frac = rng.uniform(0, 1, (natom, 3))
    if natom > 1:  # a site planted near another, possibly across a cell boundary
        frac[-1] = (frac[0] + rng.normal(0, 0.03, 3)) % 1.0
    symm = [(np.eye(3), np.zeros(3))]
    for _ in range(int(rng.integers(0, 4))):
        qm, _r = np.linalg.qr(rng.normal(size=(3, 3)))
        symm.append((qm, rng.choice([0.0, 0.5], 3)))
    ncell = tuple(int(c) for c in rng.integers(1, 5, 3))
    occ = rng.choice([0.0, 1.0], natom, p=[0.2, 0.8])
    ncopy = int(rng.integers(1, 4))
    r_copy = rng.uniform(-30, 30, (ncopy, 3))
    cf = [np.linalg.qr(rng.normal(size=(3, 3)))[0] for _ in range(ncopy)]
    kw = dict(r_copy=r_copy, cf=cf)
    if rng.random() < 0.5:
        kw["rcut"] = float(rng.uniform(3, 15))
    if rng.random() < 0.3:
        kw["rcut_copies"] = float(rng.uniform(10, 50))
    return Block.crystal(e, frac, natom_el, ids, ncell, symm=symm, occ=occ, centered=bool(rng.random() < 0.5), **kw)


@needs_reference
@pytest.mark.parametrize("seed", range(40))
def test_random_draw_free_blocks_match_reference(seed):
    b = random_draw_free_block(seed)
    xo, nao = oracle().build_atoms([b], 4, seed=seed)
    xr, nar = reference().calc_atoms([b], 4)
    assert np.array_equal(nao, nar)
    assert same(xo, xr)
