"""Structure blocks for the GPU builder (xns_build_atoms) and the rearrangement correction
(xns_rearrangement_int).

Block mirrors the fields of the reference's block class (typedefs.h:198-278) that block::calcAtoms
(CalcFunctions.cpp:251-392) reads, after the XML reader prepared them (ReadXML.cpp:254-323): site and
symmetry coordinates Cartesian, sites sorted by element, copy rotations as matrices.  Block.crystal
does that preparation for the common case of a unit cell given in fractional coordinates.
RearrBlock holds what RearrangementInt (CalcFunctions.cpp:469-545) reads of a block.
"""
import ctypes as C

import numpy as np

_p = C.c_void_p
_u32 = C.c_uint32
_i32 = C.c_int32
_dbl = C.c_double


class BlockStruct(C.Structure):
    """struct xns_block (include/xns_b200.h)."""
    _fields_ = [("natom", _u32), ("nid", _u32), ("nsymm", _u32), ("ncopy", _u32), ("ncell", _u32 * 3),
                ("cutoff", _i32), ("cutoff_copies", _i32), ("ro_mol", _i32),
                ("natom_el", _p), ("id", _p), ("r_atom", _p), ("occ", _p), ("dev", _p), ("p_symm", _p),
                ("r_symm", _p), ("r_copy", _p), ("cf", _p),
                ("e", _dbl * 9), ("r_mean", _dbl * 3), ("rcut", _dbl), ("rcut_copies", _dbl), ("dev_mol", _dbl)]


def _f64(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))


class Block:
    """One block: sites (natom x 3, Cartesian, element-sorted), natom_el sites per block element, id the
    global element index of each block element, occupancies, displacement widths (the reference's
    dev = sqrt(Uiso)), symmetry operations (p_symm nsymm x 3 x 3, r_symm nsymm x 3 Cartesian), cell
    vectors e (rows) and counts ncell, copies (r_copy ncopy x 3, cf ncopy x 3 x 3 rotation rows),
    r_mean, the cut-off radii (None = off), the molecule displacement width and the molecule
    rotation switch."""

    def __init__(self, r_atom, natom_el, id, occ=None, dev=None, p_symm=None, r_symm=None, e=None, ncell=(1, 1, 1),
                 r_copy=None, cf=None, r_mean=(0.0, 0.0, 0.0), rcut=None, rcut_copies=None, dev_mol=0.0, ro_mol=False):
        self.r_atom = _f64(r_atom, (-1, 3))
        n = len(self.r_atom)
        self.natom_el = np.ascontiguousarray(natom_el, dtype=np.uint32)
        self.id = np.ascontiguousarray(id, dtype=np.uint32)
        self.occ = _f64(np.ones(n) if occ is None else occ, (n,))
        self.dev = _f64(np.zeros(n) if dev is None else dev, (n,))
        self.p_symm = _f64(np.eye(3)[None] if p_symm is None else p_symm, (-1, 3, 3))
        self.r_symm = _f64(np.zeros((len(self.p_symm), 3)) if r_symm is None else r_symm, (-1, 3))
        self.e = _f64(np.eye(3) if e is None else e, (3, 3))
        self.ncell = tuple(int(c) for c in ncell)
        self.r_copy = _f64(np.zeros((1, 3)) if r_copy is None else r_copy, (-1, 3))
        self.cf = _f64(np.eye(3)[None].repeat(len(self.r_copy), 0) if cf is None else cf, (-1, 3, 3))
        self.r_mean = _f64(r_mean, (3,))
        self.rcut = rcut
        self.rcut_copies = rcut_copies
        self.dev_mol = float(dev_mol)
        self.ro_mol = bool(ro_mol)
        if len(self.r_symm) != len(self.p_symm) or len(self.cf) != len(self.r_copy):
            raise ValueError("Block: p_symm / r_symm and r_copy / cf must have matching lengths")
        if int(self.natom_el.sum()) != n or len(self.natom_el) != len(self.id):
            raise ValueError("Block: natom_el must sum to the number of sites and match id")

    @property
    def natom(self):
        return len(self.r_atom)

    @classmethod
    def crystal(cls, e, sites, natom_el, id, ncell, symm=None, occ=None, dev=None, centered=False, **kw):
        """A unit cell given as cell vectors e (3 x 3 rows) and fractional sites, with symmetry operations
        symm = [(rotation 3 x 3 acting on Cartesian sites, fractional translation 3)] (default: identity).
        Converted as the reference's redefAtoms / redefSymm do (CalcFunctions.cpp:116-133); centered sets
        r_mean to the mean of all replicated sites (block::calcMean, :140-160)."""
        e = _f64(e, (3, 3))
        frac = _f64(sites, (-1, 3))
        r = frac[:, 0:1] * e[0] + frac[:, 1:2] * e[1] + frac[:, 2:3] * e[2]
        if symm is None:
            symm = [(np.eye(3), np.zeros(3))]
        p = np.array([np.asarray(s[0], dtype=np.float64) for s in symm])
        t = np.array([np.asarray(s[1], dtype=np.float64) for s in symm])
        rs = t[:, 0:1] * e[0] + t[:, 1:2] * e[1] + t[:, 2:3] * e[2]
        r_mean = kw.pop("r_mean", (0.0, 0.0, 0.0))
        if centered:
            pos = np.einsum("skl,al->ask", p, r) + rs[None]
            nc = np.asarray(ncell)
            g = np.stack(np.meshgrid(*[np.arange(c) for c in nc], indexing="ij"), -1).reshape(-1, 3)
            shifts = g @ e
            r_mean = (pos.reshape(-1, 3)[:, None, :] + shifts[None]).reshape(-1, 3).mean(0)
        return cls(r, natom_el, id, occ=occ, dev=dev, p_symm=p, r_symm=rs, e=e, ncell=ncell, r_mean=r_mean, **kw)

    def as_struct(self):
        """(BlockStruct, arrays it points into): keep the second alive while the struct is used."""
        s = BlockStruct()
        s.natom, s.nid, s.nsymm, s.ncopy = self.natom, len(self.id), len(self.p_symm), len(self.r_copy)
        s.ncell[:] = list(self.ncell)
        s.cutoff = int(self.rcut is not None)
        s.cutoff_copies = int(self.rcut_copies is not None)
        s.ro_mol = int(self.ro_mol)
        keep = [self.natom_el, self.id, self.r_atom, self.occ, self.dev, self.p_symm, self.r_symm, self.r_copy, self.cf]
        (s.natom_el, s.id, s.r_atom, s.occ, s.dev, s.p_symm, s.r_symm, s.r_copy,
         s.cf) = [a.ctypes.data_as(_p) for a in keep]
        s.e[:] = list(self.e.ravel())
        s.r_mean[:] = list(self.r_mean)
        s.rcut = 0.0 if self.rcut is None else float(self.rcut)
        s.rcut_copies = 0.0 if self.rcut_copies is None else float(self.rcut_copies)
        s.dev_mol = self.dev_mol
        return s, keep


def block_array(blocks):
    """A C array of BlockStruct for a list of blocks, and the arrays to keep alive."""
    arr = (BlockStruct * max(1, len(blocks)))()
    keep = []
    for i, b in enumerate(blocks):
        arr[i], k = b.as_struct()
        keep.append(k)
    return arr, keep


class RearrBlockStruct(C.Structure):
    """struct xns_rearr_block (include/xns_b200.h)."""
    _fields_ = [("natom", _u32), ("nid", _u32), ("rearrangement", _u32), ("coeff", _u32), ("natom_el", _p), ("id", _p),
                ("r_atom", _p), ("neighb_off", _p), ("neighb_r", _p), ("neighb_id", _p), ("rcorr", _dbl)]


class RearrBlock:
    """A block as RearrangementInt (CalcFunctions.cpp:469-545) reads it: sites (natom x 3, element-sorted),
    natom_el, global element ids, per site a list of (x, y, z, global element) neighbours from the
    block's Rearrangement file, Rcorr, and coeff = Ncopy * Ncell.x * Ncell.y * Ncell.z * Nsymm."""

    def __init__(self, r_atom, natom_el, id, neighbours, rcorr, coeff, rearrangement=True):
        self.r_atom = _f64(r_atom, (-1, 3))
        self.natom_el = np.ascontiguousarray(natom_el, dtype=np.uint32)
        self.id = np.ascontiguousarray(id, dtype=np.uint32)
        if len(neighbours) != len(self.r_atom):
            raise ValueError("RearrBlock: one neighbour list per site")
        self.neighb_off = np.ascontiguousarray(np.concatenate([[0], np.cumsum([len(n) for n in neighbours])]),
                                               dtype=np.uint32)
        flat = [t for n in neighbours for t in n]
        self.neighb_r = _f64([t[:3] for t in flat] if flat else np.zeros((0, 3)), (-1, 3))
        self.neighb_id = np.ascontiguousarray([int(t[3]) for t in flat], dtype=np.uint32)
        self.rcorr = float(rcorr)
        self.coeff = int(coeff)
        self.rearrangement = bool(rearrangement)

    def as_struct(self, struct=RearrBlockStruct):
        s = struct()
        s.natom, s.nid, s.rearrangement, s.coeff = len(self.r_atom), len(self.id), int(self.rearrangement), self.coeff
        keep = [self.natom_el, self.id, self.r_atom, self.neighb_off, self.neighb_r, self.neighb_id]
        s.natom_el, s.id, s.r_atom, s.neighb_off, s.neighb_r, s.neighb_id = [a.ctypes.data_as(_p) for a in keep]
        s.rcorr = self.rcorr
        return s, keep


def rearr_block_array(blocks, struct=RearrBlockStruct):
    arr = (struct * max(1, len(blocks)))()
    keep = []
    for i, b in enumerate(blocks):
        arr[i], k = b.as_struct(struct)
        keep.append(k)
    return arr, keep
