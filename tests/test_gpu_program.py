"""GPU end to end: the reference program built from its sources (oracle/_ref/XaNSoNS_OMP) and the same
program relinked against the drop-in calc functions (softx-d-16-00083_b200/lib/XaNSoNS_B200: the
reference's main.cpp, ReadXML.cpp and IO.cpp unchanged) run the same XML decks; their output files
must agree -- PDF files byte for byte, intensity files within the relative tolerance."""
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


def write_deck(d, name, scenario, elements, names, calc_extra, calc_children):
    with open(os.path.join(d, "atoms.txt"), "w") as f:
        for nm, xyz in zip(names, elements):
            for x, y, z in xyz:
                f.write("%s %.17g %.17g %.17g\n" % (nm, x, y, z))
    with open(os.path.join(d, "sl.txt"), "w") as f:
        f.write("# element scattering length\nNa 3.63\nCl 9.58\nPt 7.63\n")
    with open(os.path.join(d, name + ".xml"), "w") as f:
        f.write('<?xml version="1.0"?>\n<Main>\n  <Calculation name="%s" source="neutron" scenario="%s" '
                'FFfilename="sl.txt" %s>\n%s\n  </Calculation>\n  <Block>\n    <Atoms filename="atoms.txt"/>\n'
                '  </Block>\n</Main>\n' % (name, scenario, calc_extra, calc_children))


def run_both(tmp_path, name):
    outs = {}
    for tag, exe in (("ref", REF_EXE), ("ours", OUR_EXE)):
        d = tmp_path / tag
        for f in os.listdir(tmp_path / "deck"):
            (d / f).write_bytes((tmp_path / "deck" / f).read_bytes())
        r = subprocess.run([exe, name + ".xml"] + (["4"] if tag == "ref" else []), cwd=d, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        outs[tag] = {f: (d / f).read_text() for f in os.listdir(d) if f.endswith(".txt") and f not in ("atoms.txt", "sl.txt")}
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
