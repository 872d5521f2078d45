"""CPU: the error bound of the histogram kernel's centred FP32 estimate (hist.cu, centred_consts and
XNS_CENTRED2), checked by emulating the kernel's float32 operation sequence in numpy on adversarial
tile pairs.  The approximate instruction (rsqrt.approx, taken as 2 ulp) gets that worst-case error
with random signs; the reference distance is taken in extended precision.

The kernel bins a pair from the estimate only when the estimate is farther than the bound from a bin
edge, so the bound holding for every pair is what keeps the histogram bit-identical to the
reference's; pairs within the bound are binned exactly in FP64."""
import numpy as np
import pytest

U = 2.0 ** -24
MAGIC = np.float32(12582912.0)
f32 = np.float32


def fma32(a, b, c):
    # a*b is exact in float64 for float32 operands; the sum is rounded once more, to float32
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(np.float32)


def centred_consts(R0, rhoI, rhoJ):
    """Mirror of centred_consts in hist.cu (float32 arithmetic, 2 % enlargement)."""
    u = f32(U)
    R0f = f32(R0)
    rhoI, rhoJ = f32(rhoI), f32(rhoJ)
    rs = rhoI + rhoJ
    rr = f32(12.0) * rhoI * rhoJ
    PQ = f32(2.0) * R0f * rs + rhoI * rhoI + rhoJ * rhoJ + R0f + f32(0.25)
    Lr = f32(1.998) * (R0f - rs) * f32(0.999999)
    F = (f32(0.5) + (R0f + f32(0.5)) / (f32(2.0) * (R0f - rs) * f32(0.999999))) * f32(1.000001)
    K1 = (f32(3.0) * F + f32(1.0)) * u * f32(1.02)
    K0 = (u * (PQ + rr) / Lr * f32(1.02) + f32(50.0) * u * u * (R0f + rs) * f32(1.02) + f32(1e-9)
          + R0f * f32(9.094947e-13))
    fl = np.floor(R0)
    R = fl + 0.5
    return dict(R2=f32(R * R), NR=f32(-R), N2R=f32(-2.0 * R), S=(R0 - R) * (R0 + R), R0i=int(fl), K1=K1,
                mc=f32(0.5) - K0 - K1 - f32(1e-6), K0=float(K0), K1d=float(K1))


def tile_radius(h, ib):
    """Mirror of pair_geom's radius: per-axis half extents (+1 bin) enlarged by 1e-6, in float32."""
    e = (h * ib + 1.0).astype(np.float32) * f32(1.000001)
    return float(np.sqrt((e.astype(np.float32) ** 2).sum(dtype=np.float32)) * f32(1.000001))


def emulate_tile_pair(rng, bin_, hI, hJ, cI, cJ, n=4000, corners=True):
    ib = 1.0 / bin_
    D = (cI - cJ) * ib
    rhoI, rhoJ = tile_radius(hI, ib), tile_radius(hJ, ib)
    R0 = np.sqrt((D ** 2).sum())
    assert R0 >= 2.0 * (rhoI + rhoJ)  # far_pair
    c = centred_consts(R0, rhoI, rhoJ)
    xi = cI + rng.uniform(-1, 1, (n, 3)) * hI
    xj = cJ + rng.uniform(-1, 1, (n, 3)) * hJ
    if corners:  # a quarter of the atoms on box corners: the largest |a|, |b|
        k = n // 4
        xi[:k] = cI + rng.choice([-1.0, 1.0], (k, 3)) * hI
        xj[:k] = cJ + rng.choice([-1.0, 1.0], (k, 3)) * hJ
    a = (xi - cI) * ib
    b = (xj - cJ) * ib
    P = (2.0 * (a @ D) + (a * a).sum(1) + c["S"]).astype(np.float32)
    Q = (2.0 * (b @ D) - (b * b).sum(1)).astype(np.float32)
    A32 = a.astype(np.float32)
    B32 = (f32(-2.0) * b.astype(np.float32)).astype(np.float32)
    # per pair (a row of I against a row of J)
    pq = (P - Q).astype(np.float32)
    ab = fma32(A32[:, 0], B32[:, 0], fma32(A32[:, 1], B32[:, 1], (A32[:, 2] * B32[:, 2]).astype(np.float32)))
    num = (pq + ab).astype(np.float32)
    d2 = (num + c["R2"]).astype(np.float32)
    e1 = rng.choice([-3.9, 3.9], n) * U
    y = ((1.0 / np.sqrt(d2.astype(np.float64))) * (1.0 + e1)).astype(np.float32)
    t0 = fma32(d2, y, c["NR"])
    res = fma32(t0, (c["N2R"] - t0).astype(np.float32), num)
    t = fma32(res, (y * f32(0.5)).astype(np.float32), t0)
    tm = (t + MAGIC).astype(np.float32)
    d = (t - (tm - MAGIC).astype(np.float32)).astype(np.float32)
    fast = np.abs(d) <= fma32(np.abs(t), -c["K1"], c["mc"])
    nround = (tm.view(np.int32) - MAGIC.view(np.int32)).astype(np.int64)
    # reference distance in extended precision
    dx = (xi.astype(np.longdouble) - xj.astype(np.longdouble)) * np.longdouble(ib)
    r = np.sqrt((dx * dx).sum(1))
    target = r - np.longdouble(c["R0i"]) - np.longdouble(0.5)
    err = np.abs(t.astype(np.longdouble) - target).astype(np.float64)
    bound = c["K0"] + c["K1d"] * (np.abs(t.astype(np.float64)) + 1.0)
    return err, bound, fast, nround, np.floor(r).astype(np.int64) - c["R0i"], R0


def test_centred_bound_holds_and_fast_bins_are_exact():
    rng = np.random.default_rng(7)
    bin_ = 0.001
    worst, nfast, ntot = 0.0, 0, 0
    for trial in range(300):
        hI = rng.uniform(1.0, 8.0, 3)
        hJ = rng.uniform(1.0, 8.0, 3)
        rho = tile_radius(hI, 1.0 / bin_) + tile_radius(hJ, 1.0 / bin_)
        # from the far threshold up to 3e5 bins, half of them right at the threshold
        R0 = 2.0 * rho * (1.0 + 1e-9) if trial % 2 == 0 else rng.uniform(2.0 * rho, max(3e5, 2.5 * rho))
        v = rng.normal(size=3)
        cJ = rng.uniform(-50, 50, 3)
        cI = cJ + v / np.linalg.norm(v) * R0 * bin_
        err, bound, fast, nround, want, _ = emulate_tile_pair(rng, bin_, hI, hJ, cI, cJ)
        worst = max(worst, float(np.max(err / bound)))
        assert np.all(err <= bound), (trial, float(np.max(err / bound)))
        assert np.array_equal(nround[fast], want[fast]), trial
        nfast += int(fast.sum())
        ntot += fast.size
    assert worst < 1.0
    # the bound is useful: most pairs are binned from the estimate
    assert nfast / ntot > 0.9


@pytest.mark.parametrize("R0_bins", [1.2e5, 2.9e5])
def test_centred_near_fraction_at_benchmark_distances(R0_bins):
    """At 1e5-bin distances and tiles of the benchmark's size (about 6.8 A half extents at 0.001 A bins)
    the centred estimate sends about one percent of the pairs to the exact path (the direct estimate's
    margin, 6u r, sends 8 to 20 %)."""
    rng = np.random.default_rng(11)
    bin_ = 0.001
    fr = []
    for _ in range(20):
        hI = np.full(3, 6.8)
        hJ = np.full(3, 6.8)
        v = rng.normal(size=3)
        cJ = rng.uniform(-50, 50, 3)
        cI = cJ + v / np.linalg.norm(v) * R0_bins * bin_
        err, bound, fast, _, _, _ = emulate_tile_pair(rng, bin_, hI, hJ, cI, cJ, corners=False)
        assert np.all(err <= bound)
        fr.append(1.0 - fast.mean())
    assert np.mean(fr) < 0.02
