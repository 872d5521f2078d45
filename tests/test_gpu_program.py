"""GPU end to end: the reference program built from its sources (oracle/_ref/XaNSoNS_OMP) and the same
program relinked against the drop-in (softx-d-16-00083_b200/lib/XaNSoNS_B200: the reference's main.cpp,
ReadXML.cpp, IO.cpp and CalcFunctions.cpp sources, its calc functions, structure builder, rearrangement
correction and writers replaced by the GPU library's) run the same XML decks; their output files
must agree -- PDF and atom files byte for byte, intensity files within the relative tolerance."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

from xns_b200 import synth

pytestmark = pytest.mark.gpu

REF_EXE = os.path.join(ROOT, "oracle", "_ref", "XaNSoNS_OMP")
OUR_EXE = os.path.join(ROOT, "softx-d-16-00083_b200", "lib", "XaNSoNS_B200")

need_exes = pytest.mark.skipif(not (os.path.exists(REF_EXE) and os.path.exists(OUR_EXE)),
                               reason="reference program or relinked program not built")


def write_deck(d, name, scenario, elements, names, calc_extra, calc_children, block_extra=""):
    with open(os.path.join(d, "atoms.txt"), "w") as f:
        for nm, xyz in zip(names, elements):
            for x, y, z in xyz:
                f.write("%s %.17g %.17g %.17g\n" % (nm, x, y, z))
    with open(os.path.join(d, "sl.txt"), "w") as f:
        f.write("# element scattering length\nNa 3.63\nCl 9.58\nPt 7.63\n")
    with open(os.path.join(d, name + ".xml"), "w") as f:
        f.write('<?xml version="1.0"?>\n<Main>\n  <Calculation name="%s" source="neutron" scenario="%s" '
                'FFfilename="sl.txt" %s>\n%s\n  </Calculation>\n  <Block>\n    <Atoms filename="atoms.txt"/>\n'
                '%s  </Block>\n</Main>\n' % (name, scenario, calc_extra, calc_children, block_extra))


def run_both(tmp_path, name):
    outs = {}
    for tag, exe in (("ref", REF_EXE), ("ours", OUR_EXE)):
        d = tmp_path / tag
        for f in os.listdir(tmp_path / "deck"):
            (d / f).write_bytes((tmp_path / "deck" / f).read_bytes())
        r = subprocess.run([exe, name + ".xml"] + (["4"] if tag == "ref" else []), cwd=d, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        outs[tag] = {f: (d / f).read_text() for f in os.listdir(d)
                     if (f.endswith(".txt") or f.endswith(".xyz")) and f not in ("atoms.txt", "sl.txt", "neigh.txt")}
    assert sorted(outs["ref"]) == sorted(outs["ours"]) and outs["ref"]
    return outs


def table(text):
    return np.array([[float(v) for v in line.split()] for line in text.strip().splitlines()])


def make_dirs(tmp_path):
    for t in ("deck", "ref", "ours"):
        (tmp_path / t).mkdir()
    return str(tmp_path / "deck")


@need_exes
def test_program_debye_pdf(tmp_path):
    els = synth.rocksalt_cube(cells=6, seed=31)
    write_deck(make_dirs(tmp_path), "rs", "DebyePDF", els, ["Na", "Cl"], 'hist_bin="0.001"',
               '    <q min="0.1" max="25" N="512"/>\n    <PDF type="rPDF" PrintPartial="yes"/>')
    outs = run_both(tmp_path, "rs")
    for f, text in outs["ref"].items():
        if "PDF" in f:
            assert text == outs["ours"][f], f  # PDF: bit-identical values, identical files
        else:
            a, b = table(text), table(outs["ours"][f])
            assert np.array_equal(a[:, 0], b[:, 0])
            assert np.max(np.abs(a[:, 1] - b[:, 1]) / np.abs(a[:, 1])) < 1e-5, f


@need_exes
def test_program_debye(tmp_path):
    els = synth.fcc_sphere(n=1500, seed=32)
    write_deck(make_dirs(tmp_path), "sp", "Debye", els, ["Pt"], "", '    <q min="0.1" max="10" N="1024"/>')
    outs = run_both(tmp_path, "sp")
    for f, text in outs["ref"].items():
        a, b = table(text), table(outs["ours"][f])
        assert np.array_equal(a[:, 0], b[:, 0])
        assert np.max(np.abs(a[:, 1] - b[:, 1]) / np.abs(a[:, 1])) < 1e-5, f


@need_exes
def test_program_2d(tmp_path):
    els = synth.rocksalt_cube(cells=3, seed=33)
    write_deck(make_dirs(tmp_path), "p2", "2D", els, ["Na", "Cl"], 'wavelength="0.5"',
               '    <q min="0.5" max="6" N="32" Nfi="24"/>\n    <Euler min="0 0 0" max="90 45 30" N="2 1 2" convention="ZYX"/>')
    outs = run_both(tmp_path, "p2")
    for f, text in outs["ref"].items():
        a, b = table(text), table(outs["ours"][f])
        assert a.shape == b.shape
        if "2D" in f:
            floor = 1e-2 * np.median(np.abs(a))
            assert np.max(np.abs(a - b) / np.maximum(np.abs(a), floor)) < 1e-5, f
        else:
            assert np.max(np.abs(a[:, 1] - b[:, 1]) / np.abs(a[:, 1])) < 1e-5, f


@need_exes
def test_program_debye_rearrangement_and_atoms(tmp_path):
    """a molecule with a Rearrangement file (RearrangementInt after the Debye sum) and PrintAtoms
    (the builder's atoms written by printAtoms): intensities within 1e-5, the atom file byte for byte"""
    from test_rearrangement import molecule_block
    mb = molecule_block(n=60, seed=4, coeff=1, rcorr=0.4)
    names = ["Na", "Cl"]
    ne = [int(v) for v in mb.natom_el]
    els = [mb.r_atom[:ne[0]], mb.r_atom[ne[0]:]]
    d = make_dirs(tmp_path)
    with open(os.path.join(d, "neigh.txt"), "w") as f:
        for i in range(len(mb.r_atom)):
            lo, hi = int(mb.neighb_off[i]), int(mb.neighb_off[i + 1])
            f.write("%d %d\n" % (i, hi - lo))
            for k in range(lo, hi):
                x, y, z = mb.neighb_r[k]
                f.write("%s %.17g %.17g %.17g\n" % (names[int(mb.neighb_id[k])], x, y, z))
    write_deck(d, "mol", "Debye", els, names, 'PrintAtoms="yes"', '    <q min="0.1" max="12" N="400"/>',
               '    <Rearrangement filename="neigh.txt" Rcorr="0.4"/>\n')
    outs = run_both(tmp_path, "mol")
    assert any(f.endswith(".xyz") for f in outs["ref"])
    for f, text in outs["ref"].items():
        if f.endswith(".xyz"):
            assert text == outs["ours"][f], f
        else:
            a, b = table(text), table(outs["ours"][f])
            assert np.array_equal(a[:, 0], b[:, 0])
            assert np.max(np.abs(a[:, 1] - b[:, 1]) / np.abs(a[:, 1])) < 1e-5, f
