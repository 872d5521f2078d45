"""CPU: the oracle restatement (oracle/xns_oracle.c) is pinned against the golden vectors that the
reference's own calc functions produced (tests/golden/make_golden.py), and, where the reference
build is present, against the reference on further seeded inputs."""
import os

import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_err, split_elements

from xns_b200 import synth

HAVE_REF = os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                                       "libxnsref.so"))


@pytest.mark.parametrize("name", golden_names("hist"))
def test_hist_bitexact(oracle, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    assert oracle.hist_size(els, float(g["bin"])) == int(g["nhist"])
    h = oracle.hist(els, int(g["nhist"]), float(g["bin"]))
    assert np.array_equal(h, g["hist"])
    assert oracle.atomic_density(els) == float(g["p0"])


@pytest.mark.parametrize("name", golden_names("debye"))
def test_debye(oracle, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    # the full-size pattern (5000 atoms x 1024 q) on every 64th q, so that the CPU suite stays short
    sub = slice(None, None, 64 if len(g["q"]) > 256 else 1)
    I = oracle.int_debye(els, g["q"][sub], int(g["source"]), ff=None if g.get("ff") is None else g["ff"][:, sub],
                         sl=g.get("sl"), polar=bool(g["polar"]), lam=float(g["lam"]))
    assert rel_err(I, g["I"][sub]) < 1e-12


def test_partial_debye(oracle):
    g = load_golden("partial__rocksalt_3blocks")
    els = split_elements(g["xyz"], g["n_el"])
    I = oracle.int_partial_debye(els, g["n_el_block"], g["q"], int(g["source"]), sl=g["sl"])
    assert rel_err(I, g["I"]) < 1e-12


@pytest.mark.parametrize("name", golden_names("pdf"))
def test_pdf_bitexact_and_iq(oracle, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    nh, bin = int(g["nhist"]), float(g["bin"])
    h = oracle.hist(els, nh, bin)
    pdf = oracle.pdf(h, g["n_el"], nh, bin, int(g["pdftype"]), float(g["p0"]), g["sl"])
    assert np.array_equal(pdf, g["pdf"])
    I = oracle.int_1d_hist(h, g["n_el"], nh, bin, g["q"], 0, sl=g["sl"])
    assert rel_err(I, g["I"]) < 1e-12


def test_iq_from_hist_xray(oracle):
    g = load_golden("iqhist__rocksalt_xray")
    I = oracle.int_1d_hist(g["hist"], g["n_el"], int(g["nhist"]), float(g["bin"]), g["q"], 1, ff=g["ff"], polar=True,
                           lam=float(g["lam"]))
    assert rel_err(I, g["I"]) < 1e-12


@pytest.mark.parametrize("name", golden_names("2d"))
def test_2d(oracle, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    I2D, I = oracle.int_2d(els, g["q"], int(g["nfi"]), g["emin"], g["emax"], g["en"], int(g["conv"]), float(g["lam"]),
                           int(g["source"]), ff=g.get("ff"), sl=g.get("sl"), polar=bool(g["polar"]))
    assert rel_err(I2D, g["I2D"]) < 1e-12
    assert rel_err(I, g["I"]) < 1e-12


def test_rotation_conventions(oracle):
    g = load_golden("rot__all")
    for c in range(12):
        assert np.allclose(oracle.rot_matrix(g["euler"], c), g["m"][c], rtol=0, atol=1e-15)


def test_known_answer_two_atoms(oracle):
    """Two atoms at distance r: I(q) = b^2 (1 + sin(qr)/(qr + 1e-8)) (N = 2)."""
    r = 2.5
    q = synth.q_mesh(0.1, 10, 64)
    I = oracle.int_debye([np.array([[0, 0, 0], [r, 0, 0]], float)], q, 0, sl=[2.0])
    assert rel_err(I, 4.0 * (1 + np.sin(q * r) / (q * r + 1e-8))) < 1e-14


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_oracle_vs_reference_seeded():
    from oracle import Oracle, Reference
    O, R = Oracle(), Reference(threads=4)
    els = synth.rocksalt_cube(cells=4, seed=101)
    for bin in (0.001, 0.0137):
        nh = R.hist_size(els, bin)
        assert np.array_equal(O.hist(els, nh, bin), R.hist(els, nh, bin))
    q = synth.q_mesh(0.3, 15, 96)
    assert rel_err(O.int_debye(els, q, 0, sl=[1.0, -2.0]), R.int_debye(els, q, 0, sl=[1.0, -2.0])) < 1e-11


def test_mlp_oracle_gradients_by_finite_differences():
    """The perceptron oracle's analytic gradient against central differences (FP64, BF16 weights held
    fixed by perturbing only the biases and a few BF16-exact weight steps)."""
    import mlp_oracle
    dims = (5, 7, 6, 3)
    rng = np.random.default_rng(0)
    n = 7 * 5 + 7 + 6 * 7 + 6 + 3 * 6 + 3
    p = rng.normal(size=n).astype(np.float32)
    x, t = rng.normal(size=(4, 5)), rng.normal(size=(4, 3))
    w = np.array([1.0, 2.0, 0.5])
    loss, g = mlp_oracle.gradients(p, dims, x, t, w)
    # biases are used in FP64 as given: perturb them directly
    bias_idx = list(range(35, 42)) + list(range(84, 90)) + list(range(108, 111))
    for i in bias_idx:
        e = np.zeros(n)
        e[i] = 1e-4
        lp, _ = mlp_oracle.gradients(p.astype(np.float64) + e, dims, x, t, w)
        lm, _ = mlp_oracle.gradients(p.astype(np.float64) - e, dims, x, t, w)
        assert abs((lp - lm) / 2e-4 - g[i]) < 1e-6 * max(1.0, abs(g[i]))
    # weights go through BF16 rounding: step by exactly one BF16 ulp of 1.0 on weights equal to 1.0
    q = p.copy()
    for i in (0, 50, 95):
        q[i] = 1.0
    _, gq = mlp_oracle.gradients(q, dims, x, t, w)
    for i in (0, 50, 95):
        h = 2.0 ** -7
        qp, qm = q.copy(), q.copy()
        qp[i], qm[i] = 1.0 + h, 1.0 - h
        lp, _ = mlp_oracle.gradients(qp, dims, x, t, w)
        lm, _ = mlp_oracle.gradients(qm, dims, x, t, w)
        assert abs((lp - lm) / (2 * h) - gq[i]) < 2e-2 * max(1.0, abs(gq[i]))
