"""CPU: the output writers (xns_write_*) byte for byte against the reference's own writers
(printI, printPartialI, printI2, printPDF, printPartialPDF, printAtoms, IO.cpp:51-167, 273-295)
compiled from its sources.  The writers are host code: no GPU needed."""
import os

import numpy as np
import pytest

import xns_b200
from oracle import REF_SO, Reference

pytestmark = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")

EDGE = np.array([0.0, -0.0, 1.0, -1.0, 0.5, 1e-300, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
                 -1.7976931348623157e308, np.inf, -np.inf, np.nan, 9.9999995e-5, 9.9999994999999999e-5, 1.0000005,
                 1.00000049999999, 123456.75, 0.1, 1 / 3, 2 / 3, 99999995.0, 99999994.99999999, 1e22, 1e23])


def values(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(n) * 10.0 ** rng.integers(-30, 30, n)
    v[:len(EDGE)] = EDGE
    # decimal near-ties at 7 significant digits: d.dddddd5 x 10^k, as close as binary allows
    k = rng.integers(-20, 20, 200)
    v[len(EDGE):len(EDGE) + 200] = (rng.integers(1000000, 9999999, 200) + 0.5) * 10.0 ** (k - 6)
    return v


def same_file(a, b):
    with open(a, "rb") as fa, open(b, "rb") as fb:
        return fa.read() == fb.read()


def test_print_i(tmp_path):
    R = Reference()
    q, I = values(20000, 1), values(20000, 2)
    assert R.print_i(str(tmp_path / "ref"), q, I, 1) == 0
    xns_b200.write_i(str(tmp_path / "ours.txt"), q, I)
    assert same_file(tmp_path / "ref_xray_1D.txt", tmp_path / "ours.txt")


def test_print_partial_i(tmp_path):
    R = Reference()
    nq, nb = 512, 3
    q, I = values(nq, 3), values(nq * 6, 4)
    assert R.print_partial_i(str(tmp_path / "ref"), q, I, 0, nb) == 0
    c = 0
    for ib in range(nb):
        for jb in range(ib, nb):
            xns_b200.write_i(str(tmp_path / "ours.txt"), q, I[c * nq:(c + 1) * nq])
            assert same_file(tmp_path / ("ref_neut_%d-%d_1D.txt" % (ib, jb)), tmp_path / "ours.txt")
            c += 1


def test_print_i2(tmp_path):
    R = Reference()
    I2 = values(300 * 257, 5).reshape(300, 257)
    assert R.print_i2(str(tmp_path / "ref"), I2, 0) == 0
    xns_b200.write_i2(str(tmp_path / "ours.txt"), I2)
    assert same_file(tmp_path / "ref_neut_2D.txt", tmp_path / "ours.txt")


@pytest.mark.parametrize("tail", ["zeros", "tiny_negative", "none", "all_zero"])
def test_print_pdf_and_partials(tmp_path, tail):
    R = Reference()
    nh, bin_ = 5000, 0.01
    names = ["Cl", "Na"]
    pdf = values(3 * nh, 6)
    for c in range(3):
        seg = pdf[c * nh:(c + 1) * nh]
        if tail == "zeros":
            seg[4000:] = 0.0
        elif tail == "tiny_negative":
            seg[3000:] = -5e-10  # kept by |value| in the total, dropped in the partials
        elif tail == "all_zero":
            seg[:] = 0.0
    assert R.print_pdf(str(tmp_path / "ref"), pdf[:nh], bin_, 1, 2) == 0
    xns_b200.write_pdf(str(tmp_path / "ours.txt"), pdf[:nh], bin_)
    assert same_file(tmp_path / "ref_xray_rPDF.txt", tmp_path / "ours.txt")
    assert R.print_partial_pdf(str(tmp_path / "ref"), pdf, nh, bin_, 1, 1, names) == 0
    c = 0
    for i in range(2):
        for j in range(i, 2):
            xns_b200.write_pdf(str(tmp_path / "ours.txt"), pdf[c * nh:(c + 1) * nh], bin_, partial=True)
            assert same_file(tmp_path / ("ref_xray_partial_PDF_%s_%s.txt" % (names[i], names[j])), tmp_path / "ours.txt")
            c += 1


def test_print_atoms(tmp_path):
    R = Reference()
    els = [values(3 * 7000, 7).reshape(-1, 3), np.zeros((0, 3)), values(3 * 5000, 8).reshape(-1, 3)]
    names = ["Ag", "C", "Zn"]  # the reference's ID map order (sorted names)
    assert R.print_atoms(str(tmp_path / "ref"), els, names) == 0
    xns_b200.write_atoms(str(tmp_path / "ours.xyz"), els, names)
    assert same_file(tmp_path / "ref_atoms.xyz", tmp_path / "ours.xyz")


def test_unwritable_path_is_an_error(tmp_path):
    with pytest.raises(OSError):
        xns_b200.write_i(str(tmp_path / "missing_dir" / "x.txt"), [1.0], [2.0])
