"""Test infrastructure only: ctypes access to the checkers.

    Oracle()      the FP64 C restatement (oracle/liboracle.so, built from xns_oracle.c)
    Reference()   the reference's own CPU calc functions compiled from its sources
                  (oracle/_ref/libxnsref.so, built by oracle/Makefile where the sources exist)

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module, as the checker or the
timed CPU baseline; the product never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libxnsref.so")

_p = C.c_void_p
_u32 = C.c_uint32
_dbl = C.c_double
_int = C.c_int


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


def _flat(elements):
    arrs = [np.ascontiguousarray(e, dtype=np.float64).reshape(-1, 3) for e in elements]
    n_el = np.array([len(a) for a in arrs], dtype=np.uint32)
    xyz = np.ascontiguousarray(np.concatenate(arrs) if len(arrs) else np.zeros((0, 3)))
    return xyz, n_el


def _ff(ff, nq):
    return None if ff is None else np.ascontiguousarray(np.asarray(ff, dtype=np.float64).reshape(-1, nq))


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class _BlockStruct(C.Structure):
    """xo_block / the harness's xr_block: the same layout as the library's xns_block."""
    _fields_ = [("natom", _u32), ("nid", _u32), ("nsymm", _u32), ("ncopy", _u32), ("ncell", _u32 * 3),
                ("cutoff", C.c_int32), ("cutoff_copies", C.c_int32), ("ro_mol", C.c_int32),
                ("natom_el", _p), ("id", _p), ("r_atom", _p), ("occ", _p), ("dev", _p), ("p_symm", _p),
                ("r_symm", _p), ("r_copy", _p), ("cf", _p),
                ("e", _dbl * 9), ("r_mean", _dbl * 3), ("rcut", _dbl), ("rcut_copies", _dbl), ("dev_mol", _dbl)]


def _blocks(blocks):
    """C array of block descriptions from objects with the attributes of xns_b200.structure.Block."""
    arr = (_BlockStruct * max(1, len(blocks)))()
    keep = []
    for i, b in enumerate(blocks):
        s = arr[i]
        a = [np.ascontiguousarray(b.natom_el, dtype=np.uint32), np.ascontiguousarray(b.id, dtype=np.uint32)] + [
            np.ascontiguousarray(x, dtype=np.float64) for x in (b.r_atom, b.occ, b.dev, b.p_symm, b.r_symm, b.r_copy, b.cf)]
        keep.append(a)
        s.natom, s.nid, s.nsymm, s.ncopy = len(a[2]), len(a[1]), len(a[5]), len(a[7])
        s.ncell[:] = [int(c) for c in b.ncell]
        s.cutoff, s.cutoff_copies, s.ro_mol = int(b.rcut is not None), int(b.rcut_copies is not None), int(b.ro_mol)
        s.natom_el, s.id, s.r_atom, s.occ, s.dev, s.p_symm, s.r_symm, s.r_copy, s.cf = [x.ctypes.data_as(_p) for x in a]
        s.e[:] = [float(v) for v in np.asarray(b.e, dtype=np.float64).ravel()]
        s.r_mean[:] = [float(v) for v in b.r_mean]
        s.rcut = 0.0 if b.rcut is None else float(b.rcut)
        s.rcut_copies = 0.0 if b.rcut_copies is None else float(b.rcut_copies)
        s.dev_mol = float(b.dev_mol)
    return arr, keep


class _RearrStruct(C.Structure):
    """xo_rearr_block / the harness's xr_rearr_block: the library's xns_rearr_block layout."""
    _fields_ = [("natom", _u32), ("nid", _u32), ("rearrangement", _u32), ("coeff", _u32), ("natom_el", _p), ("id", _p),
                ("r_atom", _p), ("neighb_off", _p), ("neighb_r", _p), ("neighb_id", _p), ("rcorr", _dbl)]


def _rearr(fn, I0, q, blocks, nel, source, ff, sl, partial, polar, lam, ntot):
    """calls fn (xo_ / xnsref_rearrangement_int) on a copy of I0; blocks: objects with the attributes of
    xns_b200.structure.RearrBlock"""
    I = np.array(I0, dtype=np.float64, copy=True)
    q = _f64(q)
    arr = (_RearrStruct * max(1, len(blocks)))()
    keep = []
    for i, b in enumerate(blocks):
        a = [np.ascontiguousarray(b.natom_el, dtype=np.uint32), np.ascontiguousarray(b.id, dtype=np.uint32),
             _f64(b.r_atom), np.ascontiguousarray(b.neighb_off, dtype=np.uint32), _f64(b.neighb_r),
             np.ascontiguousarray(b.neighb_id, dtype=np.uint32)]
        keep.append(a)
        s = arr[i]
        s.natom, s.nid, s.rearrangement, s.coeff = len(a[2]), len(a[1]), int(b.rearrangement), int(b.coeff)
        s.natom_el, s.id, s.r_atom, s.neighb_off, s.neighb_r, s.neighb_id = [x.ctypes.data_as(_p) for x in a]
        s.rcorr = float(b.rcorr)
    ffm = _ff(ff, len(q))
    fn(_ptr(I), _ptr(q), len(q), C.cast(arr, _p), len(blocks), nel, source, _ptr(ffm), _ptr(_f64(sl)), int(partial),
       int(polar), lam, ntot)
    return I


def _split(ptr, n_el, free):
    tot = int(np.sum(n_el))
    flat = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(_dbl)), shape=(max(tot, 1) * 3,))[:tot * 3].copy()
    free(ptr)
    out, o = [], 0
    for n in n_el:
        out.append(flat[3 * o:3 * (o + int(n))].reshape(-1, 3))
        o += int(n)
    return out


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError("%s is not built (make -C oracle)" % path)
        L = self.lib = C.CDLL(path)
        L.xo_rot_matrix.argtypes = [_p, _u32, _p]
        L.xo_hist_size.argtypes = [_p, _p, _u32, _dbl]
        L.xo_hist_size.restype = _u32
        L.xo_atomic_density.argtypes = [_p, _p, _u32]
        L.xo_atomic_density.restype = _dbl
        L.xo_hist.argtypes = [_p, _p, _u32, _u32, _dbl, _p]
        L.xo_int_debye.argtypes = [_p, _p, _u32, _p, _u32, _int, _p, _p, _int, _dbl, _p]
        L.xo_int_partial_debye.argtypes = [_p, _p, _u32, _u32, _p, _p, _u32, _int, _p, _p, _int, _dbl, _p]
        L.xo_int_1d_hist.argtypes = [_p, _p, _u32, _u32, _dbl, _p, _u32, _int, _p, _p, _int, _dbl, _p]
        L.xo_pdf.argtypes = [_p, _p, _u32, _u32, _dbl, _int, _dbl, _p, _p]
        L.xo_int_2d.argtypes = [_p, _p, _u32, _p, _u32, _u32, _p, _p, _p, _u32, _dbl, _int, _p, _p, _int, _p, _p]
        L.xo_rearrangement_int.argtypes = [_p, _p, _u32, _p, _u32, _u32, _int, _p, _p, _int, _int, _dbl, _u32]
        L.xo_build_atoms.argtypes = [_p, _u32, _u32, C.c_uint64, _p, _p]
        L.xo_build_atoms.restype = _p
        L.xo_free.argtypes = [_p]
        L.xo_philox.argtypes = [_p, _p, _p]
        L.xo_amp_plane.argtypes = [_p, _p, _u32, _dbl, _dbl, _u32, _dbl, _dbl, _u32, _int, _p, _p, _p]

    def rearrangement_int(self, I0, q, blocks, nel, source, ff=None, sl=None, partial=False, polar=False, lam=0.0, ntot=0):
        return _rearr(self.lib.xo_rearrangement_int, I0, q, blocks, nel, source, ff, sl, partial, polar, lam, ntot)

    def philox(self, ctr, key):
        c, k, o = np.array(ctr, dtype=np.uint32), np.array(key, dtype=np.uint32), np.zeros(4, dtype=np.uint32)
        self.lib.xo_philox(_ptr(c), _ptr(k), _ptr(o))
        return o

    def build_atoms(self, blocks, nel, seed=0):
        """(list of per-element (n, 3) arrays, n_all) from xo_build_atoms."""
        arr, keep = _blocks(blocks)
        n_el = np.zeros(nel, dtype=np.uint32)
        n_all = np.zeros(max(1, sum(len(b.id) for b in blocks)), dtype=np.uint32)
        ptr = self.lib.xo_build_atoms(C.cast(arr, _p), len(blocks), nel, seed, _ptr(n_el), _ptr(n_all))
        del keep
        return _split(ptr, n_el, self.lib.xo_free), n_all[:sum(len(b.id) for b in blocks)]

    def rot_matrix(self, euler, convention):
        e = _f64(euler)
        m = np.zeros(9)
        self.lib.xo_rot_matrix(_ptr(e), convention, _ptr(m))
        return m.reshape(3, 3)

    def hist_size(self, elements, bin):
        xyz, n = _flat(elements)
        return self.lib.xo_hist_size(_ptr(xyz), _ptr(n), len(n), bin)

    def atomic_density(self, elements):
        xyz, n = _flat(elements)
        return self.lib.xo_atomic_density(_ptr(xyz), _ptr(n), len(n))

    def hist(self, elements, nhist, bin):
        xyz, n = _flat(elements)
        out = np.zeros(len(n) * (len(n) + 1) // 2 * nhist, dtype=np.uint64)
        if self.lib.xo_hist(_ptr(xyz), _ptr(n), len(n), nhist, bin, _ptr(out)):
            raise ValueError("pair distance beyond nhist")
        return out

    def int_debye(self, elements, q, source, ff=None, sl=None, polar=False, lam=0.0):
        xyz, n = _flat(elements)
        q = _f64(q)
        out = np.zeros(len(q))
        self.lib.xo_int_debye(_ptr(xyz), _ptr(n), len(n), _ptr(q), len(q), source, _ptr(_ff(ff, len(q))), _ptr(_f64(sl)),
                              int(polar), lam, _ptr(out))
        return out

    def int_partial_debye(self, elements, n_el_block, q, source, ff=None, sl=None, polar=False, lam=0.0):
        xyz, n = _flat(elements)
        neb = np.ascontiguousarray(n_el_block, dtype=np.uint32)
        nb = neb.shape[1]
        q = _f64(q)
        out = np.zeros((1 + nb * (nb + 1) // 2) * len(q))
        self.lib.xo_int_partial_debye(_ptr(xyz), _ptr(n), len(n), nb, _ptr(neb), _ptr(q), len(q), source,
                                      _ptr(_ff(ff, len(q))), _ptr(_f64(sl)), int(polar), lam, _ptr(out))
        return out

    def int_1d_hist(self, hist, n_el, nhist, bin, q, source, ff=None, sl=None, polar=False, lam=0.0):
        h = np.ascontiguousarray(hist, dtype=np.uint64)
        n = np.ascontiguousarray(n_el, dtype=np.uint32)
        q = _f64(q)
        out = np.zeros(len(q))
        self.lib.xo_int_1d_hist(_ptr(h), _ptr(n), len(n), nhist, bin, _ptr(q), len(q), source, _ptr(_ff(ff, len(q))),
                                _ptr(_f64(sl)), int(polar), lam, _ptr(out))
        return out

    def pdf(self, hist, n_el, nhist, bin, pdftype, p0, sl):
        h = np.ascontiguousarray(hist, dtype=np.uint64)
        n = np.ascontiguousarray(n_el, dtype=np.uint32)
        P = len(n) * (len(n) + 1) // 2
        out = np.zeros((1 + P) * nhist)
        self.lib.xo_pdf(_ptr(h), _ptr(n), len(n), nhist, bin, pdftype, p0, _ptr(_f64(sl)), _ptr(out))
        return out

    def int_2d(self, elements, q, nfi, euler_min, euler_max, euler_n, convention, lam, source, ff=None, sl=None,
               polar=False):
        xyz, n = _flat(elements)
        q = _f64(q)
        I2D = np.zeros((len(q), nfi))
        I = np.zeros(len(q))
        en = np.ascontiguousarray(euler_n, dtype=np.uint32)
        self.lib.xo_int_2d(_ptr(xyz), _ptr(n), len(n), _ptr(q), len(q), nfi, _ptr(_f64(euler_min)), _ptr(_f64(euler_max)),
                           _ptr(en), convention, lam, source, _ptr(_ff(ff, len(q))), _ptr(_f64(sl)), int(polar), _ptr(I2D),
                           _ptr(I))
        return I2D, I

    def amp_plane(self, elements, qx0, dqx, nqx, qy0, dqy, nqy, source, coef=None, sl=None):
        xyz, n = _flat(elements)
        out = np.zeros((nqy, nqx))
        self.lib.xo_amp_plane(_ptr(xyz), _ptr(n), len(n), qx0, dqx, nqx, qy0, dqy, nqy, source,
                              _ptr(_f64(coef)), _ptr(_f64(sl)), _ptr(out))
        return out


class Reference:
    """The reference's own calc functions (CalcFunctions.cpp) behind oracle/ref_harness.cpp."""

    def __init__(self, path=REF_SO, threads=None):
        if not os.path.exists(path):
            raise FileNotFoundError("%s is not built (make -C oracle ref, needs the reference sources)" % path)
        self.threads = threads or os.cpu_count() or 1
        L = self.lib = C.CDLL(path)
        L.xnsref_rot_matrix.argtypes = [_p, _u32, _p]
        L.xnsref_calc_atoms.argtypes = [_p, _u32, _u32, _p, _p]
        L.xnsref_calc_atoms.restype = _p
        L.xnsref_free.argtypes = [_p]
        L.xnsref_rearrangement_int.argtypes = [_p, _p, _u32, _p, _u32, _u32, _int, _p, _p, _int, _int, _dbl, _u32]
        L.xnsref_print_i.argtypes = [C.c_char_p, _p, _p, _u32, _u32]
        L.xnsref_print_partial_i.argtypes = [C.c_char_p, _p, _p, _u32, _u32, _u32]
        L.xnsref_print_i2.argtypes = [C.c_char_p, _p, _u32, _u32, _u32]
        L.xnsref_print_pdf.argtypes = [C.c_char_p, _p, _u32, _dbl, _u32, _u32]
        L.xnsref_print_partial_pdf.argtypes = [C.c_char_p, _p, _u32, _dbl, _u32, _u32, _u32, _p]
        L.xnsref_print_atoms.argtypes = [C.c_char_p, _p, _p, _u32, _p]
        L.xnsref_hist_size.argtypes = [_p, _p, _u32, _dbl]
        L.xnsref_hist_size.restype = _u32
        L.xnsref_atomic_density.argtypes = [_p, _p, _u32]
        L.xnsref_atomic_density.restype = _dbl
        L.xnsref_calc_hist.argtypes = [_p, _p, _u32, _u32, _dbl, _int, _p]
        L.xnsref_calc_int_debye.argtypes = [_p, _p, _u32, _p, _u32, _int, _p, _p, _int, _dbl, _int, _p]
        L.xnsref_calc_int_partial_debye.argtypes = [_p, _p, _u32, _u32, _p, _p, _u32, _int, _p, _p, _int, _dbl, _int, _p]
        L.xnsref_calc_int_1d_hist.argtypes = [_p, _p, _u32, _u32, _dbl, _p, _u32, _int, _p, _p, _int, _dbl, _int, _p]
        L.xnsref_calc_pdf_and_debye.argtypes = [_p, _p, _u32, _u32, _dbl, _int, _int, _dbl, _p, _u32, _int, _p, _p, _int,
                                                _dbl, _int, _p, _p]
        L.xnsref_calc_int_2d.argtypes = [_p, _p, _u32, _p, _u32, _u32, _p, _p, _p, _u32, _dbl, _int, _p, _p, _int, _int,
                                         _p, _p]

    def rearrangement_int(self, I0, q, blocks, nel, source, ff=None, sl=None, partial=False, polar=False, lam=0.0, ntot=0):
        return _rearr(self.lib.xnsref_rearrangement_int, I0, q, blocks, nel, source, ff, sl, partial, polar, lam, ntot)

    # the reference's writers: name is the path prefix; they return the reference's status
    def print_i(self, name, q, I, source):
        q, I = _f64(q), _f64(I)
        return self.lib.xnsref_print_i(name.encode(), _ptr(q), _ptr(I), len(q), source)

    def print_partial_i(self, name, q, I, source, nblocks):
        q, I = _f64(q), _f64(I)
        return self.lib.xnsref_print_partial_i(name.encode(), _ptr(q), _ptr(I), len(q), source, nblocks)

    def print_i2(self, name, I2D, source):
        a = np.ascontiguousarray(I2D, dtype=np.float64)
        return self.lib.xnsref_print_i2(name.encode(), _ptr(a), a.shape[0], a.shape[1], source)

    def print_pdf(self, name, pdf, bin, source, pdftype):
        a = _f64(pdf)
        return self.lib.xnsref_print_pdf(name.encode(), _ptr(a), len(a), bin, source, pdftype)

    @staticmethod
    def _names(names):
        nm = [n.encode() for n in names]
        return (C.c_char_p * max(1, len(nm)))(*nm)

    def print_partial_pdf(self, name, pdf, nhist, bin, source, pdftype, names):
        a = _f64(pdf)
        return self.lib.xnsref_print_partial_pdf(name.encode(), _ptr(a), nhist, bin, source, pdftype, len(names),
                                                 C.cast(self._names(names), _p))

    def print_atoms(self, name, elements, names):
        xyz, n = _flat(elements)
        return self.lib.xnsref_print_atoms(name.encode(), _ptr(xyz), _ptr(n), len(n), C.cast(self._names(names), _p))

    def calc_atoms(self, blocks, nel):
        """(list of per-element (n, 3) arrays, n_all) from the reference's own block::calcAtoms."""
        arr, keep = _blocks(blocks)
        n_el = np.zeros(nel, dtype=np.uint32)
        n_all = np.zeros(max(1, sum(len(b.id) for b in blocks)), dtype=np.uint32)
        ptr = self.lib.xnsref_calc_atoms(C.cast(arr, _p), len(blocks), nel, _ptr(n_el), _ptr(n_all))
        del keep
        return _split(ptr, n_el, self.lib.xnsref_free), n_all[:sum(len(b.id) for b in blocks)]

    def rot_matrix(self, euler, convention):
        e = _f64(euler)
        m = np.zeros(9)
        self.lib.xnsref_rot_matrix(_ptr(e), convention, _ptr(m))
        return m.reshape(3, 3)

    def hist_size(self, elements, bin):
        xyz, n = _flat(elements)
        return self.lib.xnsref_hist_size(_ptr(xyz), _ptr(n), len(n), bin)

    def atomic_density(self, elements):
        xyz, n = _flat(elements)
        return self.lib.xnsref_atomic_density(_ptr(xyz), _ptr(n), len(n))

    def hist(self, elements, nhist, bin):
        xyz, n = _flat(elements)
        out = np.zeros(len(n) * (len(n) + 1) // 2 * nhist, dtype=np.uint64)
        self.lib.xnsref_calc_hist(_ptr(xyz), _ptr(n), len(n), nhist, bin, self.threads, _ptr(out))
        return out

    def int_debye(self, elements, q, source, ff=None, sl=None, polar=False, lam=0.0):
        xyz, n = _flat(elements)
        q = _f64(q)
        out = np.zeros(len(q))
        self.lib.xnsref_calc_int_debye(_ptr(xyz), _ptr(n), len(n), _ptr(q), len(q), source, _ptr(_ff(ff, len(q))),
                                       _ptr(_f64(sl)), int(polar), lam, self.threads, _ptr(out))
        return out

    def int_partial_debye(self, elements, n_el_block, q, source, ff=None, sl=None, polar=False, lam=0.0):
        xyz, n = _flat(elements)
        neb = np.ascontiguousarray(n_el_block, dtype=np.uint32)
        nb = neb.shape[1]
        q = _f64(q)
        out = np.zeros((1 + nb * (nb + 1) // 2) * len(q))
        self.lib.xnsref_calc_int_partial_debye(_ptr(xyz), _ptr(n), len(n), nb, _ptr(neb), _ptr(q), len(q), source,
                                               _ptr(_ff(ff, len(q))), _ptr(_f64(sl)), int(polar), lam, self.threads,
                                               _ptr(out))
        return out

    def int_1d_hist(self, hist, n_el, nhist, bin, q, source, ff=None, sl=None, polar=False, lam=0.0):
        h = np.ascontiguousarray(hist, dtype=np.uint64)
        n = np.ascontiguousarray(n_el, dtype=np.uint32)
        q = _f64(q)
        out = np.zeros(len(q))
        self.lib.xnsref_calc_int_1d_hist(_ptr(h), _ptr(n), len(n), nhist, bin, _ptr(q), len(q), source,
                                         _ptr(_ff(ff, len(q))), _ptr(_f64(sl)), int(polar), lam, self.threads, _ptr(out))
        return out

    def pdf_and_debye(self, elements, nhist, bin, scenario, pdftype, p0, q, source, ff=None, sl=None, polar=False,
                      lam=0.0):
        xyz, n = _flat(elements)
        P = len(n) * (len(n) + 1) // 2
        q = _f64(q) if q is not None else np.zeros(1)
        I = np.zeros(len(q))
        pdf = np.zeros((1 + P) * nhist)
        self.lib.xnsref_calc_pdf_and_debye(_ptr(xyz), _ptr(n), len(n), nhist, bin, scenario, pdftype, p0, _ptr(q), len(q),
                                           source, _ptr(_ff(ff, len(q))), _ptr(_f64(sl)), int(polar), lam, self.threads,
                                           _ptr(I), _ptr(pdf))
        return I, pdf

    def int_2d(self, elements, q, nfi, euler_min, euler_max, euler_n, convention, lam, source, ff=None, sl=None,
               polar=False):
        xyz, n = _flat(elements)
        q = _f64(q)
        I2D = np.zeros((len(q), nfi))
        I = np.zeros(len(q))
        en = np.ascontiguousarray(euler_n, dtype=np.uint32)
        self.lib.xnsref_calc_int_2d(_ptr(xyz), _ptr(n), len(n), _ptr(q), len(q), nfi, _ptr(_f64(euler_min)),
                                    _ptr(_f64(euler_max)), _ptr(en), convention, lam, source, _ptr(_ff(ff, len(q))),
                                    _ptr(_f64(sl)), int(polar), self.threads, _ptr(I2D), _ptr(I))
        return I2D, I
