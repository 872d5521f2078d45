"""Python binding of the xns_b200 C ABI (include/xns_b200.h) over ctypes.

The library is the in-tree build softx-d-16-00083_b200/lib/libxns_b200.so, loaded at the first call
into it (importing the package alone maps nothing); a missing build raises ImportError there, and every
call raises XnsError on a non-zero status.  There is no CPU code path here: each function calls the
CUDA library.

Arrays follow the reference's layout (see the header): coordinates per element as (n_e, 3) float64
arrays, element pairs a <= b in loop order, histograms element-pair major.
"""
import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libxns_b200.so")

NEUTRON, XRAY = 0, 1
RDF, PDF, RPDF = 0, 1, 2
DEBYE_HIST, PDF_ONLY, DEBYE_PDF = 2, 3, 4


class XnsError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("xns status %d: %s" % (status, msg))
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("xns_b200: %s is not built (run softx-d-16-00083_b200/build.py)" % LIB_PATH)
    return C.CDLL(LIB_PATH)


_p = C.c_void_p
_u32 = C.c_uint32
_dbl = C.c_double
_int = C.c_int
_PP = C.POINTER(C.c_void_p)


def _declare(lib):
    """The C prototypes of the entry points (include/xns_b200.h)."""
    lib.xns_create.argtypes = [_int, C.POINTER(_p)]
    lib.xns_destroy.argtypes = [_p]
    lib.xns_destroy.restype = None
    lib.xns_last_error.argtypes = [_p]
    lib.xns_last_error.restype = C.c_char_p
    lib.xns_status_string.argtypes = [_int]
    lib.xns_status_string.restype = C.c_char_p
    lib.xns_set_stream.argtypes = [_p, _p]
    lib.xns_set_memory_limit.argtypes = [_p, C.c_uint64]
    lib.xns_inject_pipeline_stall.argtypes = [_p, C.c_uint64]
    lib.xns_debye_tensor_cores.argtypes = [_p, _int]
    lib.xns_last_kernel_ms.argtypes = [_p]
    lib.xns_last_kernel_ms.restype = _dbl
    lib.xns_kernel_launches.argtypes = [_p]
    lib.xns_kernel_launches.restype = C.c_uint64
    lib.xns_calc_hist.argtypes = [_p, _PP, _p, _u32, _u32, _dbl, _p]
    lib.xns_calc_int_1d_hist.argtypes = [_p, _p, _p, _u32, _u32, _dbl, _p, _u32, _int, _PP, _p, _int, _dbl, _p]
    lib.xns_calc_pdf.argtypes = [_p, _p, _p, _u32, _u32, _dbl, _int, _dbl, _p, _p]
    lib.xns_calc_pdf_and_debye.argtypes = [_p, _PP, _p, _u32, _u32, _dbl, _int, _int, _dbl, _p, _u32, _int, _PP, _p, _int,
                                           _dbl, _p, _p, _p]
    lib.xns_calc_int_debye.argtypes = [_p, _PP, _p, _u32, _p, _u32, _int, _PP, _p, _int, _dbl, _p]
    lib.xns_calc_int_partial_debye.argtypes = [_p, _PP, _p, _u32, _u32, _p, _p, _u32, _int, _PP, _p, _int, _dbl, _p]
    lib.xns_calc_int_2d.argtypes = [_p, _PP, _p, _u32, _p, _u32, _u32, _p, _p, _p, _u32, _dbl, _int, _PP, _p, _int, _p, _p]
    lib.xns_hist_transform_bf16x3.argtypes = [_p, _p, _u32, _u32, _dbl, _p, _u32, _p]
    lib.xns_hist_transform_exact.argtypes = [_p, _p, _u32, _u32, _dbl, _p, _u32, _p]
    lib.xns_hist_transform_split.argtypes = [_p, _p, _u32, _u32, _dbl, _p, _u32, _p]
    _BATCH_IN = [_u32, _p, _p, _p, _u32, _dbl, _p, _u32, _int, _PP, _p, _int, _dbl]
    lib.xns_calc_batch_debye_hist.argtypes = [_p] + _BATCH_IN + [_p, _p]
    lib.xns_batch_create.argtypes = [_p] + _BATCH_IN + [_int, C.POINTER(_p)]
    lib.xns_batch_run.argtypes = [_p, _p, _p]
    lib.xns_batch_last_ms.argtypes = [_p]
    lib.xns_batch_last_ms.restype = _dbl
    lib.xns_batch_last_error.argtypes = [_p]
    lib.xns_batch_last_error.restype = C.c_char_p
    lib.xns_batch_tuning.argtypes = [_p, C.POINTER(_u32), C.POINTER(_u32)]
    lib.xns_batch_tuning.restype = _dbl
    lib.xns_batch_destroy.argtypes = [_p]
    lib.xns_batch_destroy.restype = None
    lib.xns_mlp_create.argtypes = [_p, _p, C.c_uint64, C.POINTER(_p)]
    lib.xns_mlp_destroy.argtypes = [_p]
    lib.xns_mlp_destroy.restype = None
    lib.xns_mlp_last_error.argtypes = [_p]
    lib.xns_mlp_last_error.restype = C.c_char_p
    lib.xns_mlp_param_count.argtypes = [_p]
    lib.xns_mlp_param_count.restype = C.c_long
    lib.xns_mlp_get_params.argtypes = [_p, _p]
    lib.xns_mlp_set_params.argtypes = [_p, _p]
    lib.xns_mlp_forward.argtypes = [_p, _p, _int, _p]
    lib.xns_mlp_gradients.argtypes = [_p, _p, _p, _p, _int, _p, C.POINTER(_dbl)]
    lib.xns_mlp_train.argtypes = [_p, _p, _p, _p, _int, _int, _int, C.c_float, C.POINTER(_dbl)]
    lib.xns_calc_amp_plane.argtypes = [_p, _PP, _p, _u32, _dbl, _dbl, _u32, _dbl, _dbl, _u32, _int, _p, _p, _p]
    lib.xns_binning_features.argtypes = [_p, _p, _u32, _p]
    lib.xns_binning_correction.argtypes = [_p, _p, _p, _u32, _dbl, _p, _u32, _dbl, _p]
    lib.xns_build_atoms.argtypes = [_p, _p, _u32, _u32, C.c_uint64, _p, _p, C.POINTER(_p)]
    lib.xns_copy_atoms.argtypes = [_p, _PP]
    lib.xns_rearrangement_int.argtypes = [_p, _p, _p, _u32, _p, _u32, _u32, _int, _PP, _p, _int, _int, _dbl, _u32]
    lib.xns_calc_hist_passes.argtypes = [_p, _PP, _p, _u32, _u32, _dbl, C.c_uint64, _p]
    lib.xns_write_i.argtypes = [C.c_char_p, _p, _p, _u32]
    lib.xns_write_i2.argtypes = [C.c_char_p, _p, _u32, _u32]
    lib.xns_write_pdf.argtypes = [C.c_char_p, _p, _u32, _dbl, _int]
    lib.xns_write_atoms.argtypes = [C.c_char_p, _p, _p, _u32, _PP]
    lib.xns_pdf_and_debye_device.argtypes = [_p, _p, _p, _u32, _u32, _dbl, _int, _int, _dbl, _p, _u32, _int, _PP, _p, _int,
                                             _dbl, _p, _p, _p]


class _Lib:
    """The CUDA library, loaded and its prototypes declared at the first call through it, so that
    importing the package (for its structure generators, say) maps no shared library; a missing build
    raises ImportError at that first call."""
    _cdll = None

    def __getattr__(self, name):
        if _Lib._cdll is None:
            cdll = _load()
            _declare(cdll)
            _Lib._cdll = cdll
        return getattr(_Lib._cdll, name)


lib = _Lib()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


class _Elements:
    """Keeps per-element contiguous float64 (n, 3) arrays alive and exposes the pointer table."""

    def __init__(self, els):
        self.arrays = [np.ascontiguousarray(e, dtype=np.float64).reshape(-1, 3) for e in els]
        self.n_el = np.array([len(a) for a in self.arrays], dtype=np.uint32)
        self.table = (C.c_void_p * len(self.arrays))(*[a.ctypes.data for a in self.arrays])
        self.nel = len(self.arrays)
        self.ntot = int(self.n_el.sum())


def _rows(rows, nq):
    """Per-element rows (X-ray form factors) -> pointer table; None stays None."""
    if rows is None:
        return None, None
    arrs = [np.ascontiguousarray(r, dtype=np.float64).reshape(nq) for r in rows]
    return arrs, (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class _Ensemble:
    """Flattens structures (each a list of per-element (n, 3) arrays) and their per-element weights into
    the batch ABI's arrays."""

    def __init__(self, structures, q, sl=None, ff=None):
        self.nel = np.array([len(s) for s in structures], dtype=np.uint32)
        arrs = [np.ascontiguousarray(e, dtype=np.float64).reshape(-1, 3) for s in structures for e in s]
        self.n_el = np.array([len(a) for a in arrs], dtype=np.uint32)
        self.xyz = np.ascontiguousarray(np.concatenate(arrs, axis=0) if arrs else np.zeros((0, 3)))
        self.P = [int(n) * (int(n) + 1) // 2 for n in self.nel]
        self.classes = sum(self.P)
        self.q = _f64(q)
        self.sl = None if sl is None else np.ascontiguousarray(np.concatenate([np.atleast_1d(w) for w in sl]), np.float64)
        self.ffa, self.fft = (None, None) if ff is None else _rows([row for s in ff for row in s], len(self.q))

    def args(self, nhist, bin, source, polar, lam):
        return (len(self.nel), _ptr(self.nel), _ptr(self.n_el), _ptr(self.xyz), nhist, bin, _ptr(self.q), len(self.q),
                source, self.fft, _ptr(self.sl), int(polar), lam)


class Batch:
    """A planned ensemble with its launches captured in a CUDA graph (xns_batch_create)."""

    def __init__(self, ctx, structures, nhist, bin, q, source, sl=None, ff=None, polar=False, lam=0.0, autotune=False):
        self._ens = _Ensemble(structures, q, sl, ff)
        self.nhist = nhist
        self._h = _p()
        st = lib.xns_batch_create(ctx.handle, *self._ens.args(nhist, bin, source, polar, lam), int(autotune),
                                  C.byref(self._h))
        if st:
            raise XnsError(st, lib.xns_last_error(ctx.handle).decode())

    def run(self, want_hist=False):
        I = np.zeros((len(self._ens.nel), len(self._ens.q)))
        h = np.zeros(self._ens.classes * self.nhist, dtype=np.uint64) if want_hist else None
        st = lib.xns_batch_run(self._h, _ptr(I), _ptr(h))
        if st:
            raise XnsError(st, lib.xns_batch_last_error(self._h).decode())
        return (I, h) if want_hist else I

    @property
    def last_ms(self):
        return lib.xns_batch_last_ms(self._h)

    def tuning(self):
        ct, wb = _u32(), _u32()
        ms = lib.xns_batch_tuning(self._h, C.byref(ct), C.byref(wb))
        return int(ct.value), int(wb.value), ms

    def close(self):
        if self._h:
            lib.xns_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MLP:
    """The learned correction's perceptron on the GPU (xns_mlp_*): dims = (in, hidden, hidden, out)."""

    def __init__(self, ctx, dims, seed=0):
        self.dims = tuple(int(d) for d in dims)
        d = np.array(self.dims, dtype=np.int32)
        self._h = _p()
        st = lib.xns_mlp_create(ctx.handle, _ptr(d), seed, C.byref(self._h))
        if st:
            raise XnsError(st, lib.xns_last_error(ctx.handle).decode())

    def _check(self, st):
        if st:
            raise XnsError(st, lib.xns_mlp_last_error(self._h).decode())

    @property
    def nparams(self):
        return int(lib.xns_mlp_param_count(self._h))

    def get_params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        self._check(lib.xns_mlp_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(lib.xns_mlp_set_params(self._h, _ptr(p)))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], self.dims[3]), dtype=np.float32)
        self._check(lib.xns_mlp_forward(self._h, _ptr(x), x.shape[0], _ptr(y)))
        return y

    def gradients(self, x, t, w=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_double()
        self._check(lib.xns_mlp_gradients(self._h, _ptr(x), _ptr(t), _ptr(w), x.shape[0], _ptr(g), C.byref(loss)))
        return loss.value, g

    def train(self, x, t, w=None, batch=128, epochs=1, lr=1e-3):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
        loss = C.c_double()
        self._check(lib.xns_mlp_train(self._h, _ptr(x), _ptr(t), _ptr(w), x.shape[0], batch, epochs, lr, C.byref(loss)))
        return loss.value

    def close(self):
        if self._h:
            lib.xns_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device.  Mirrors the reference's calc functions (CalcFunctions.cpp:546-1092)."""

    def __init__(self, device=-1):
        self._h = _p()
        st = lib.xns_create(device, C.byref(self._h))
        if st:
            msg = lib.xns_last_error(self._h).decode()
            lib.xns_destroy(self._h)
            self._h = None
            raise XnsError(st, msg)

    def close(self):
        if self._h:
            lib.xns_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st:
            raise XnsError(st, lib.xns_last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    @property
    def last_kernel_ms(self):
        return lib.xns_last_kernel_ms(self._h)

    @property
    def kernel_launches(self):
        return int(lib.xns_kernel_launches(self._h))

    def set_stream(self, stream_ptr):
        self._check(lib.xns_set_stream(self._h, stream_ptr))

    def inject_pipeline_stall(self, wait_limit_ns):
        """Failure-path test: the next tensor-core transform's waits run out (see the header)."""
        self._check(lib.xns_inject_pipeline_stall(self._h, int(wait_limit_ns)))

    def debye_tensor_cores(self, on):
        """Path of the exact Debye sum on a uniform q mesh: the integer tensor cores (True, the default)
        or the FP32 sine recurrence (False); see the header."""
        self._check(lib.xns_debye_tensor_cores(self._h, int(bool(on))))

    def set_memory_limit(self, nbytes):
        """Caps the calc functions' device scratch in this context (0: no cap); a call that would need
        more raises XnsError with status XNS_ERR_NOMEM (5)."""
        self._check(lib.xns_set_memory_limit(self._h, int(nbytes)))

    # -- structure builder -----------------------------------------------------------------------
    def build_atoms(self, blocks, nel, seed=0):
        """block::calcAtoms on the GPU for a list of structure.Block.  Returns (device address of the
        element-major x y z doubles, n_el per element, n_all per block element); the device array stays
        valid until the next build."""
        from .structure import block_array
        arr, keep = block_array(blocks)
        n_el = np.zeros(nel, dtype=np.uint32)
        n_all = np.zeros(max(1, sum(len(b.id) for b in blocks)), dtype=np.uint32)
        dev = _p()
        self._check(lib.xns_build_atoms(self._h, C.cast(arr, _p), len(blocks), nel, seed, _ptr(n_el), _ptr(n_all),
                                        C.byref(dev)))
        del keep
        return dev.value, n_el, n_all[:sum(len(b.id) for b in blocks)]

    def copy_atoms(self, n_el):
        """The last build's atoms as a list of (n_e, 3) float64 arrays."""
        out = [np.zeros((int(n), 3), dtype=np.float64) for n in n_el]
        table = (_p * max(1, len(out)))(*[o.ctypes.data_as(_p) for o in out])
        self._check(lib.xns_copy_atoms(self._h, C.cast(table, _PP)))
        return out

    def rearrangement_int(self, I0, q, blocks, nel, source, ff=None, sl=None, partial=False, polar=False, lam=0.0,
                          ntot=0):
        """RearrangementInt on the GPU for a list of structure.RearrBlock; returns the corrected copy of I0."""
        from .structure import rearr_block_array
        I = np.array(I0, dtype=np.float64, copy=True)
        q = _f64(q)
        arr, keep = rearr_block_array(blocks)
        ffa, fft = _rows(ff, len(q))
        self._check(lib.xns_rearrangement_int(self._h, _ptr(I), _ptr(q), len(q), C.cast(arr, _p), len(blocks), nel, source,
                                              fft, _ptr(_f64(sl)), int(partial), int(polar), lam, ntot))
        del keep, ffa
        return I

    # -- calc functions --------------------------------------------------------------------------
    def calc_hist(self, elements, nhist, bin):
        el = _Elements(elements)
        out = np.zeros(el.nel * (el.nel + 1) // 2 * nhist, dtype=np.uint64)
        self._check(lib.xns_calc_hist(self._h, el.table, _ptr(el.n_el), el.nel, nhist, bin, _ptr(out)))
        return out

    def calc_hist_passes(self, elements, nhist, bin, max_tile_pairs):
        """calc_hist taking the spatial plan's tile pairs at most max_tile_pairs per pass."""
        el = _Elements(elements)
        out = np.zeros(el.nel * (el.nel + 1) // 2 * nhist, dtype=np.uint64)
        self._check(lib.xns_calc_hist_passes(self._h, el.table, _ptr(el.n_el), el.nel, nhist, bin, max_tile_pairs,
                                             _ptr(out)))
        return out

    def calc_int_1d_hist(self, hist, n_el, nhist, bin, q, source, ff=None, sl=None, polar=False, lam=0.0):
        hist = np.ascontiguousarray(hist, dtype=np.uint64)
        n_el = np.ascontiguousarray(n_el, dtype=np.uint32)
        q = _f64(q)
        ffa, fft = _rows(ff, len(q))
        sl = _f64(sl)
        out = np.zeros(len(q))
        self._check(lib.xns_calc_int_1d_hist(self._h, _ptr(hist), _ptr(n_el), len(n_el), nhist, bin, _ptr(q), len(q),
                                             source, fft, _ptr(sl), int(polar), lam, _ptr(out)))
        return out

    def calc_pdf(self, hist, n_el, nhist, bin, pdftype, p0, sl):
        hist = np.ascontiguousarray(hist, dtype=np.uint64)
        n_el = np.ascontiguousarray(n_el, dtype=np.uint32)
        sl = _f64(sl)
        P = len(n_el) * (len(n_el) + 1) // 2
        out = np.zeros((1 + P) * nhist)
        self._check(lib.xns_calc_pdf(self._h, _ptr(hist), _ptr(n_el), len(n_el), nhist, bin, pdftype, p0, _ptr(sl),
                                     _ptr(out)))
        return out

    def calc_batch_debye_hist(self, structures, nhist, bin, q, source, sl=None, ff=None, polar=False, lam=0.0,
                              want_hist=False):
        """I(q) (nstruct x nq) of an ensemble in one pass; sl / ff are per structure, per element."""
        ens = _Ensemble(structures, q, sl, ff)
        I = np.zeros((len(ens.nel), len(ens.q)))
        h = np.zeros(ens.classes * nhist, dtype=np.uint64) if want_hist else None
        self._check(lib.xns_calc_batch_debye_hist(self._h, *ens.args(nhist, bin, source, polar, lam), _ptr(I), _ptr(h)))
        return (I, h) if want_hist else I

    def calc_amp_plane(self, elements, qx0, dqx, nqx, qy0, dqy, nqy, source, coef=None, sl=None):
        """|A(qx, qy)|^2 / N on a Cartesian plane (nqy x nqx), tensor cores with exact digit sums."""
        el = _Elements(elements)
        coef = None if coef is None else np.ascontiguousarray(coef, dtype=np.float64).reshape(-1, 9)
        sl = _f64(sl)
        out = np.zeros((nqy, nqx))
        self._check(lib.xns_calc_amp_plane(self._h, el.table, _ptr(el.n_el), el.nel, qx0, dqx, nqx, qy0, dqy, nqy, source,
                                           _ptr(coef), _ptr(sl), _ptr(out)))
        return out

    def batch(self, structures, nhist, bin, q, source, sl=None, ff=None, polar=False, lam=0.0, autotune=False):
        return Batch(self, structures, nhist, bin, q, source, sl, ff, polar, lam, autotune)

    def hist_transform(self, hist, bin, q, scheme="exact"):
        """G[c, i] = sum_k hist[c, k] sin(q_i r_k)/(q_i r_k + 1e-8): scheme "bf16x3" (split BF16 on the
        tensor cores, FP32 accumulation), "exact" (integer digits on the tensor cores, exact accumulation)
        or "split" (FP64 angle splitting, the form the calc functions use)."""
        hist = np.ascontiguousarray(np.atleast_2d(hist), dtype=np.uint64)
        q = _f64(q)
        G = np.zeros((hist.shape[0], len(q)))
        fn = {"bf16x3": lib.xns_hist_transform_bf16x3, "exact": lib.xns_hist_transform_exact,
              "split": lib.xns_hist_transform_split}[scheme]
        self._check(fn(self._h, _ptr(hist), hist.shape[0], hist.shape[1], bin, _ptr(q), len(q), _ptr(G)))
        return G

    def calc_pdf_and_debye(self, elements, nhist, bin, scenario, pdftype, p0, q, source, ff=None, sl=None, polar=False,
                           lam=0.0, want_hist=False):
        el = _Elements(elements)
        P = el.nel * (el.nel + 1) // 2
        q = _f64(q) if q is not None else np.zeros(1)
        ffa, fft = _rows(ff, len(q))
        sl = _f64(sl)
        I = np.zeros(len(q)) if scenario != PDF_ONLY else None
        pdf = np.zeros((1 + P) * nhist) if scenario != DEBYE_HIST else None
        h = np.zeros(P * nhist, dtype=np.uint64) if want_hist else None
        self._check(lib.xns_calc_pdf_and_debye(self._h, el.table, _ptr(el.n_el), el.nel, nhist, bin, scenario, pdftype,
                                               p0, _ptr(q), len(q), source, fft, _ptr(sl), int(polar), lam, _ptr(I),
                                               _ptr(pdf), _ptr(h)))
        return I, pdf, h

    def calc_int_debye(self, elements, q, source, ff=None, sl=None, polar=False, lam=0.0):
        el = _Elements(elements)
        q = _f64(q)
        ffa, fft = _rows(ff, len(q))
        sl = _f64(sl)
        out = np.zeros(len(q))
        self._check(lib.xns_calc_int_debye(self._h, el.table, _ptr(el.n_el), el.nel, _ptr(q), len(q), source, fft,
                                           _ptr(sl), int(polar), lam, _ptr(out)))
        return out

    def calc_int_partial_debye(self, elements, n_el_block, q, source, ff=None, sl=None, polar=False, lam=0.0):
        el = _Elements(elements)
        neb = np.ascontiguousarray(n_el_block, dtype=np.uint32)  # (nel, nblocks)
        nblocks = neb.shape[1]
        q = _f64(q)
        ffa, fft = _rows(ff, len(q))
        sl = _f64(sl)
        nparts = nblocks * (nblocks + 1) // 2
        out = np.zeros(((1 + nparts) if nblocks > 1 else 1) * len(q))
        self._check(lib.xns_calc_int_partial_debye(self._h, el.table, _ptr(el.n_el), el.nel, nblocks, _ptr(neb), _ptr(q),
                                                   len(q), source, fft, _ptr(sl), int(polar), lam, _ptr(out)))
        return out

    def calc_int_2d(self, elements, q, nfi, euler_min, euler_max, euler_n, convention, lam, source, ff=None, sl=None,
                    polar=False):
        el = _Elements(elements)
        q = _f64(q)
        ffa, fft = _rows(ff, len(q))
        sl = _f64(sl)
        emin, emax = _f64(euler_min), _f64(euler_max)
        en = np.ascontiguousarray(euler_n, dtype=np.uint32)
        I2D = np.zeros((len(q), nfi))
        I = np.zeros(len(q))
        self._check(lib.xns_calc_int_2d(self._h, el.table, _ptr(el.n_el), el.nel, _ptr(q), len(q), nfi, _ptr(emin),
                                        _ptr(emax), _ptr(en), convention, lam, source, fft, _ptr(sl), int(polar),
                                        _ptr(I2D), _ptr(I)))
        return I2D, I


# -- output writers (host threads; byte-identical to the reference's IO.cpp writers) ---------------------
def _wcheck(rc, path):
    if rc:
        raise OSError("xns_b200: cannot write %s" % path)


def write_i(path, q, I):
    """printI / printPartialI (IO.cpp:109-147): q<TAB>I per line, %.6e."""
    q, I = np.ascontiguousarray(q, dtype=np.float64), np.ascontiguousarray(I, dtype=np.float64)
    _wcheck(lib.xns_write_i(path.encode(), _ptr(q), _ptr(I), len(q)), path)


def write_i2(path, I2D):
    """printI2 (IO.cpp:148-167): one row per q, each value followed by a TAB."""
    a = np.ascontiguousarray(I2D, dtype=np.float64)
    _wcheck(lib.xns_write_i2(path.encode(), _ptr(a), a.shape[0], a.shape[1]), path)


def write_pdf(path, pdf, bin, partial=False):
    """printPDF (partial=False) / one element pair of printPartialPDF (IO.cpp:51-108)."""
    a = np.ascontiguousarray(pdf, dtype=np.float64)
    _wcheck(lib.xns_write_pdf(path.encode(), _ptr(a), len(a), bin, int(partial)), path)


def write_atoms(path, elements, names):
    """printAtoms (IO.cpp:273-295) for per-element (n, 3) arrays, in the order given."""
    arrs = [np.ascontiguousarray(e, dtype=np.float64).reshape(-1, 3) for e in elements]
    n_el = np.array([len(a) for a in arrs], dtype=np.uint32)
    xyz = np.ascontiguousarray(np.concatenate(arrs) if arrs else np.zeros((0, 3)))
    nm = [n.encode() for n in names]
    table = (C.c_char_p * max(1, len(nm)))(*nm)
    _wcheck(lib.xns_write_atoms(path.encode(), _ptr(xyz), _ptr(n_el), len(n_el), C.cast(table, _PP)), path)
