"""GPU parity: the CUDA library (through its C ABI) against the reference's golden vectors and the
FP64 oracle.  Histograms and PDFs must be bit-identical; intensities agree within the stated
relative tolerances (FP32 arithmetic with FP64 reductions against the reference's FP64)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_err, rel_err_floor, split_elements

from xns_b200 import synth

pytestmark = pytest.mark.gpu

TOL_I = 1e-5       # I(q) of the plain Debye / histogram paths, max relative error
TOL_2D = 1e-5      # 2D intensity, max relative error with the denominator floored at 1e-2 x median
FLOOR_2D = 1e-2


@pytest.mark.parametrize("name", golden_names("hist"))
def test_hist_golden(gpu_ctx, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    h = gpu_ctx.calc_hist(els, int(g["nhist"]), float(g["bin"]))
    assert np.array_equal(h, g["hist"])


# the 16-cell cube (90 A) at 0.001 A and the 12-cell one at 0.002 A have many tile pairs beyond the
# centred estimate's threshold (twice the sum of the tile radii, about 48 A and 24 A)
@pytest.mark.parametrize("cells,bin,seed", [(6, 0.001, 1), (8, 0.001, 2), (5, 0.0007, 3), (7, 0.01, 4), (16, 0.001, 5),
                                            (12, 0.002, 6)])
def test_hist_vs_oracle(gpu_ctx, oracle, cells, bin, seed):
    els = synth.rocksalt_cube(cells=cells, seed=seed)
    nh = synth.hist_size(els, bin)
    assert np.array_equal(gpu_ctx.calc_hist(els, nh, bin), oracle.hist(els, nh, bin))


def test_hist_sparse_element_and_sphere(gpu_ctx, oracle):
    """A 5 % substituent spreads its few atoms over the whole crystallite: its tile pairs are wider
    than the shared-memory window and take the direct path; a sphere exercises partly filled cells."""
    els = synth.fcc_crystallite(cells=9, subst=0.05, seed=6)
    nh = synth.hist_size(els, 0.001)
    assert np.array_equal(gpu_ctx.calc_hist(els, nh, 0.001), oracle.hist(els, nh, 0.001))
    sph = synth.fcc_sphere(n=6000, seed=7)
    nh = synth.hist_size(sph, 0.001)
    assert np.array_equal(gpu_ctx.calc_hist(sph, nh, 0.001), oracle.hist(sph, nh, 0.001))


def test_hist_edge_cases(gpu_ctx, oracle):
    rng = np.random.default_rng(5)
    # single atom, an empty element, identical atoms, atoms exactly on bin edges
    one = [np.array([[1.0, 2.0, 3.0]])]
    assert gpu_ctx.calc_hist(one, 4, 0.1).sum() == 0
    edge = [np.array([[0, 0, 0], [0.25, 0, 0], [0.5, 0, 0], [0.75, 0, 0], [0, 0.5, 0], [0, 0, 0]], float)]
    nh = synth.hist_size(edge, 0.25)
    assert np.array_equal(gpu_ctx.calc_hist(edge, nh, 0.25), oracle.hist(edge, nh, 0.25))
    els = [rng.normal(0, 3, (300, 3)), np.zeros((0, 3)), rng.normal(0, 3, (257, 3)), rng.normal(0, 3, (1, 3))]
    els[2][7] = els[0][3]
    nh = synth.hist_size(els, 0.003)
    assert np.array_equal(gpu_ctx.calc_hist(els, nh, 0.003), oracle.hist(els, nh, 0.003))


@pytest.mark.parametrize("a,bin", [(5.0, 0.001), (4.0, 0.0025), (5.64, 0.001)])
def test_hist_perfect_lattice(gpu_ctx, oracle, a, bin):
    """An undisplaced crystal: lattice distances a sqrt(n) / 2 fall on bin edges or within rounding of
    them for many shells (a = 5 A and 4 A make r / bin an integer in exact arithmetic), so the FP32
    estimates send whole shells to the exact path and its correctly rounded branch decides them."""
    els = synth.rocksalt_cube(cells=12, a=a, vacancy=0.0, sigma=0.0)
    nh = synth.hist_size(els, bin)
    assert np.array_equal(gpu_ctx.calc_hist(els, nh, bin), oracle.hist(els, nh, bin))


def test_hist_out_of_range_is_an_error(gpu_ctx):
    import xns_b200
    els = [np.array([[0, 0, 0], [1.0, 0, 0]])]
    with pytest.raises(xns_b200.XnsError) as e:
        gpu_ctx.calc_hist(els, 5, 0.1)  # distance 1.0 -> bin 10 >= 5
    assert e.value.status == 4


def test_hist_checksum_full_size(gpu_ctx):
    """Full configuration (rock-salt cube, 30^3 cells, ~1.94e5 atoms, 0.001 A): the counts are the
    reference's calcHist's bit for bit (SHA-256 of the u64 counts against the hash the reference's own
    code produced, tests/golden/make_golden.py); and size-independent checks -- the total count
    equals the number of pairs of each element pair, and the histogram of a permuted, shuffled copy
    is identical."""
    import hashlib
    g = load_golden("histhash__rocksalt30_seed0_b0.001")
    els = synth.rocksalt_cube(cells=30, seed=0)
    xyz = np.ascontiguousarray(np.concatenate(els), dtype="<f8")
    assert hashlib.sha256(xyz.tobytes()).hexdigest() == str(g["xyz_sha256"]), "the cube generator changed"
    nh = synth.hist_size(els, 0.001)
    assert nh == int(g["nhist"])
    h = gpu_ctx.calc_hist(els, nh, 0.001).reshape(3, nh)
    assert hashlib.sha256(np.ascontiguousarray(h, dtype="<u8").tobytes()).hexdigest() == str(g["sha256"])
    assert int(h.sum()) == int(g["total"])
    n0, n1 = len(els[0]), len(els[1])
    assert [int(x) for x in h.sum(axis=1)] == [n0 * (n0 - 1) // 2, n0 * n1, n1 * (n1 - 1) // 2]
    rng = np.random.default_rng(9)
    shuffled = [e[rng.permutation(len(e))] for e in els]
    assert np.array_equal(gpu_ctx.calc_hist(shuffled, nh, 0.001).reshape(3, nh), h)


@pytest.mark.parametrize("name", golden_names("debye"))
def test_debye_golden(gpu_ctx, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    I = gpu_ctx.calc_int_debye(els, g["q"], int(g["source"]), ff=g.get("ff"), sl=g.get("sl"), polar=bool(g["polar"]),
                               lam=float(g["lam"]))
    assert rel_err(I, g["I"]) < TOL_I


def test_debye_vs_oracle_sphere(gpu_ctx, oracle):
    els = synth.fcc_sphere(n=2000, seed=3)
    q = synth.q_mesh(0.1, 10.0, 1024)
    I = gpu_ctx.calc_int_debye(els, q, 0, sl=[7.63])
    Io = oracle.int_debye(els, q, 0, sl=[7.63])
    assert rel_err(I, Io) < TOL_I


def test_debye_nonuniform_mesh(gpu_ctx, oracle):
    els = synth.fcc_sphere(n=500, seed=4)
    q = np.sort(np.random.default_rng(1).uniform(0.05, 12, 200))
    assert rel_err(gpu_ctx.calc_int_debye(els, q, 0, sl=[1.0]), oracle.int_debye(els, q, 0, sl=[1.0])) < TOL_I


def test_partial_debye_golden(gpu_ctx):
    g = load_golden("partial__rocksalt_3blocks")
    els = split_elements(g["xyz"], g["n_el"])
    I = gpu_ctx.calc_int_partial_debye(els, g["n_el_block"], g["q"], int(g["source"]), sl=g["sl"])
    nq = len(g["q"])
    rows, want = I.reshape(-1, nq), g["I"].reshape(-1, nq)
    assert rel_err(rows[0], want[0]) < TOL_I  # the total
    # the parts are contributions to the total, and a cross-block part oscillates around zero: its
    # error is measured against the total intensity at the same q
    for r, w in zip(rows[1:], want[1:]):
        assert float(np.max(np.abs(r - w) / np.abs(want[0]))) < TOL_I


@pytest.mark.parametrize("name", golden_names("pdf"))
def test_pdf_and_debye_golden(gpu_ctx, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    I, pdf, _ = gpu_ctx.calc_pdf_and_debye(els, int(g["nhist"]), float(g["bin"]), 4, int(g["pdftype"]), float(g["p0"]),
                                           g["q"], 0, sl=g["sl"])
    assert np.array_equal(pdf, g["pdf"])
    assert rel_err(I, g["I"]) < TOL_I


def test_iq_from_hist_golden(gpu_ctx):
    g = load_golden("iqhist__rocksalt_xray")
    I = gpu_ctx.calc_int_1d_hist(g["hist"], g["n_el"], int(g["nhist"]), float(g["bin"]), g["q"], 1, ff=g["ff"],
                                 polar=True, lam=float(g["lam"]))
    assert rel_err(I, g["I"]) < TOL_I


def test_hist_iq_vs_oracle_large(gpu_ctx, oracle):
    els = synth.rocksalt_cube(cells=10, seed=21)
    nh = synth.hist_size(els, 0.001)
    q = synth.q_mesh(0.1, 25.0, 4096)
    I, pdf, h = gpu_ctx.calc_pdf_and_debye(els, nh, 0.001, 4, 2, 0.04, q, 0, sl=[3.63, 9.58], want_hist=True)
    assert np.array_equal(h, oracle.hist(els, nh, 0.001))
    assert np.array_equal(pdf, oracle.pdf(h, [len(e) for e in els], nh, 0.001, 2, 0.04, [3.63, 9.58]))
    assert rel_err(I, oracle.int_1d_hist(h, [len(e) for e in els], nh, 0.001, q, 0, sl=[3.63, 9.58])) < TOL_I


@pytest.mark.parametrize("name", golden_names("2d"))
def test_2d_golden(gpu_ctx, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    I2D, I = gpu_ctx.calc_int_2d(els, g["q"], int(g["nfi"]), g["emin"], g["emax"], g["en"], int(g["conv"]),
                                 float(g["lam"]), int(g["source"]), ff=g.get("ff"), sl=g.get("sl"), polar=bool(g["polar"]))
    assert rel_err_floor(I2D, g["I2D"], FLOOR_2D) < TOL_2D
    assert rel_err(I, g["I"]) < TOL_2D


@pytest.mark.parametrize("max_pairs", [1000, 12345, 1 << 20])
def test_hist_in_passes(gpu_ctx, oracle, max_pairs):
    """the tile pairs taken a few at a time (as for structures whose tile-pair list would not fit the
    device): the passes add up to the one-pass histogram, bit for bit"""
    els = synth.rocksalt_cube(cells=7, seed=12)
    nh = synth.hist_size(els, 0.001)
    one = gpu_ctx.calc_hist(els, nh, 0.001)
    assert np.array_equal(gpu_ctx.calc_hist_passes(els, nh, 0.001, max_pairs), one)
    assert np.array_equal(one, oracle.hist(els, nh, 0.001))
