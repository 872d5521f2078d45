"""CPU: the digit arithmetic of the tensor-core Debye sum (csrc/debye_tc.cu), emulated in numpy.

The kernel writes A = sin / cos of coarse q points as round(127 v 2^16) in three 8-bit digits (the top
one signed, the lower two unsigned: the bytes of the integer's low word) and B = (r_min / r) cos / sin
of the offsets as round(127 v 2^24) in four signed digits (a carried bias of 128 per byte), multiplies
the digit planes exactly (levels i + j <= 3 kept), and recombines S(Q_a +- b dq) = (C_sc +- C_cs) / r_min.
These tests pin each step: exact digit round trips, the truncation of the dropped levels, the unit of
the level sum, the +- recombination against sum sin(q r) / r (CalcFunctions.cpp:576-583), and the host's
choice of offsets and coarse points per warp covering the mesh."""
import numpy as np

MAGIC = 6755399441055744.0  # 1.5 * 2^52


def low_word(v, scale):
    """The low 32 bits of fma(v, scale, 1.5 * 2^52): round-to-nearest-even of v * scale, mod 2^32."""
    t = np.asarray(v, np.float64) * scale + MAGIC  # v * scale is exact for these scales (powers of 2 times 127)
    return (t.view(np.int64) & 0xFFFFFFFF).astype(np.uint32)


def digits_a(v):
    lo = low_word(v, 127.0 * 65536.0).astype(np.int64)
    d0 = ((lo >> 16) & 0xFF).astype(np.int8).astype(np.int64)  # signed top digit
    d1 = (lo >> 8) & 0xFF                                       # unsigned
    d2 = lo & 0xFF                                              # unsigned
    return d0, d1, d2


def digits_b(v):
    lo = low_word(v, 127.0 * 16777216.0).astype(np.int64)
    d = ((lo + 0x808080) & 0xFFFFFFFF) ^ 0x808080
    return [((d >> (8 * (3 - j))) & 0xFF).astype(np.uint8).astype(np.int8).astype(np.int64) for j in range(4)]


def test_digits_round_trip_exactly():
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.uniform(-1, 1, 200000), [-1.0, 1.0, 0.0, -0.0, 1e-300, -1e-12, 0.5, -0.5]])
    d0, d1, d2 = digits_a(v)
    assert d0.min() >= -127 and d0.max() <= 127 and d1.min() >= 0 and d1.max() <= 255
    np.testing.assert_array_equal(d0 * 65536 + d1 * 256 + d2, np.rint(v * 127 * 65536).astype(np.int64))
    b = digits_b(v)
    assert min(x.min() for x in b) >= -128 and max(x.max() for x in b) <= 127 and b[0].min() >= -127
    np.testing.assert_array_equal(b[0] * 2 ** 24 + b[1] * 2 ** 16 + b[2] * 2 ** 8 + b[3],
                                  np.rint(v * 127 * 2 ** 24).astype(np.int64))


def level_sum(a, b, keep=3):
    """sum over records of A digits x B digits, by level i + j <= keep, Horner in FP64 (the drain)."""
    da, db = digits_a(a), digits_b(b)
    t = np.zeros(a.shape[1:]) if a.ndim > 1 else 0.0
    for lev in range(keep + 1):
        t = t * 256.0
        for i in range(3):
            j = lev - i
            if 0 <= j < 4:
                t = t + np.sum(da[i] * db[j], axis=0).astype(np.float64)
    return t


def test_dropped_levels_and_unit():
    """Levels i + j >= 4 change a product by less than 2^-30 of its scale; the unit 1 / (127^2 2^24) turns
    the level sum into sum A B."""
    rng = np.random.default_rng(1)
    a = rng.uniform(-1, 1, (128, 1))
    b = rng.uniform(-1, 1, (128, 1))
    s = level_sum(a, b) / (127.0 * 127.0 * 2 ** 24)
    exact = float(np.sum(a * b))
    assert abs(s - exact) < 128 * (0.5 / (127 * 65536) + 0.5 / (127 * 2 ** 24) + 2.0 ** -30)
    # every level sum of a 256-unit chunk (32768 records) stays an exact int32
    assert 32768 * 255 * 128 < 2 ** 31


def choose(nq):
    """The host's choice (debye_tc.cu): offsets |b| <= H, PA coarse points per generator warp, q tiles."""
    if nq > 64 * 31:
        return 15, 8, (nq + 64 * 31 - 1) // (64 * 31)
    best, H, PA = None, 15, 8
    for h in range(1, 16):
        na = (nq + 2 * h) // (2 * h + 1)
        pa = (na + 7) // 8
        if pa > 8:
            continue
        cost = 16 * pa + 2 * (h + 1)
        if best is None or cost < best:
            best, H, PA = cost, h, pa
    return H, PA, 1


def test_coarse_points_cover_the_mesh():
    for nq in list(range(2, 3000)) + [4096, 8192, 20000]:
        H, PA, MT = choose(nq)
        assert 1 <= H <= 15 and 1 <= PA <= 8
        assert MT * 64 * (2 * H + 1) >= nq if MT > 1 else 8 * PA * (2 * H + 1) >= nq
    assert choose(1024) == (13, 5, 1)  # 40 coarse points x 27 q: 108 values per record


def test_recombination_reproduces_the_sinc_sum():
    """S(q_k) = sum_r sin(q_k r) / r on a uniform mesh from the digit products of the coarse-point and
    offset sines, within the digits' resolution (the kernel's arithmetic, records in one chunk)."""
    rng = np.random.default_rng(2)
    r = rng.uniform(2.5, 40.0, 3000)
    q0, nq = 0.1, 1024
    dq = 9.9 / nq
    H, PA, _ = choose(nq)
    span, ncoarse = 2 * H + 1, 8 * PA
    rmin = r.min() * (1 - 1e-12)
    a = np.arange(ncoarse)
    Q = q0 + (a * span + H) * dq                                 # coarse points
    bq = np.arange(H + 1) * dq                                   # offsets
    A_sin, A_cos = np.sin(np.outer(Q, r)), np.cos(np.outer(Q, r))  # (ncoarse, records)
    s = rmin / r
    B_cos, B_sin = np.cos(np.outer(bq, r)) * s, np.sin(np.outer(bq, r)) * s  # (H + 1, records)
    unit = 1.0 / (127.0 * 127.0 * 2 ** 24 * rmin)
    C_sc = np.array([[level_sum(A_sin[i][:, None], B_cos[j][:, None])[0] for j in range(H + 1)] for i in range(ncoarse)])
    C_cs = np.array([[level_sum(A_cos[i][:, None], B_sin[j][:, None])[0] for j in range(H + 1)] for i in range(ncoarse)])
    S = np.zeros(nq)
    for k in range(nq):
        i, bb = divmod(k, span)
        bb -= H
        S[k] = (C_sc[i, abs(bb)] + (C_cs[i, abs(bb)] if bb >= 0 else -C_cs[i, abs(bb)])) * unit
    q = q0 + np.arange(nq) * dq
    exact = np.sin(np.outer(q, r)) @ (1.0 / r)
    scale = np.sum(1.0 / r)  # the sum of the terms' sizes
    assert np.max(np.abs(S - exact)) < 1e-7 * scale
