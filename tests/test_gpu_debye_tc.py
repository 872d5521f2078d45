"""GPU: the exact Debye double sum on the integer tensor cores (csrc/debye_tc.cu, the default for uniform
q meshes) against the reference's golden vectors, the FP64 oracle and the FP32 sine-recurrence path
(xns_debye_tensor_cores(ctx, 0)).  The tensor-core path carries every term to ~6e-8 of its size and
sums digit products exactly, so it must meet the reference tolerance everywhere and be the more
accurate of the two at the deepest minimum of the 5000-atom sphere (CalcFunctions.cpp:576-583)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_err, split_elements

import xns_b200
from xns_b200 import shard, synth

pytestmark = pytest.mark.gpu

TOL_I = 1e-5


@pytest.fixture
def path(gpu_ctx, request):
    """Runs the test with the tensor-core path on or off, and restores the default afterwards."""
    gpu_ctx.debye_tensor_cores(request.param)
    yield request.param
    gpu_ctx.debye_tensor_cores(True)


@pytest.mark.parametrize("path", [True, False], indirect=True, ids=["tensor", "fp32"])
@pytest.mark.parametrize("name", golden_names("debye"))
def test_debye_golden_both_paths(gpu_ctx, path, name):
    g = load_golden(name)
    els = split_elements(g["xyz"], g["n_el"])
    I = gpu_ctx.calc_int_debye(els, g["q"], int(g["source"]), ff=g.get("ff"), sl=g.get("sl"), polar=bool(g["polar"]),
                               lam=float(g["lam"]))
    assert rel_err(I, g["I"]) < TOL_I


def test_tensor_path_more_accurate_at_config1(gpu_ctx):
    """5000-atom fcc sphere, 1024 q in [0.1, 10): the sum cancels to 1e-5 of its terms at q = 0.284."""
    g = load_golden("debye__fcc5000_neutron")
    els = synth.fcc_sphere(n=5000, a=4.078, sigma=0.05, seed=0)
    assert np.array_equal(g["xyz"], np.concatenate(els))
    q = synth.q_mesh(0.1, 10.0, 1024)
    try:
        gpu_ctx.debye_tensor_cores(False)
        e32 = rel_err(gpu_ctx.calc_int_debye(els, q, xns_b200.NEUTRON, sl=[7.63]), g["I"])
        gpu_ctx.debye_tensor_cores(True)
        etc = rel_err(gpu_ctx.calc_int_debye(els, q, xns_b200.NEUTRON, sl=[7.63]), g["I"])
    finally:
        gpu_ctx.debye_tensor_cores(True)
    assert etc < 3e-6 and etc < e32


@pytest.mark.parametrize("nq,qmax", [(1024, 10.0), (100, 8.0), (2500, 12.0), (31, 3.0), (2, 1.0)])
def test_tensor_path_vs_oracle_two_elements_xray(gpu_ctx, oracle, nq, qmax):
    """Two elements, X-ray form factors and the polarisation factor; 2500 q need two q tiles of 64 coarse
    points, 2 q the smallest offset range."""
    els = synth.fcc_crystallite(cells=5, subst=0.3, seed=nq)
    q = synth.q_mesh(0.05, qmax, nq)
    ff = [1.0 + 8.0 * np.exp(-0.05 * q * q), 1.0 + 15.0 * np.exp(-0.03 * q * q)]
    I = gpu_ctx.calc_int_debye(els, q, xns_b200.XRAY, ff=ff, polar=True, lam=1.54)
    Io = oracle.int_debye(els, q, xns_b200.XRAY, ff=ff, polar=True, lam=1.54)
    assert rel_err(I, Io) < TOL_I


def test_tensor_path_q_zero_on_mesh(gpu_ctx, oracle):
    """q = 0 on the mesh: the reference's sin(0)/(0 + 1e-8) = 0 for every pair."""
    els = synth.fcc_sphere(n=400, seed=7)
    q = np.linspace(0.0, 6.0, 200)
    assert rel_err(gpu_ctx.calc_int_debye(els, q, 0, sl=[7.63]), oracle.int_debye(els, q, 0, sl=[7.63])) < TOL_I


def test_close_pair_falls_back_to_fp32_path(gpu_ctx):
    """A pair 1e-3 A apart puts r_max / r_min above 2^8: the call takes the FP32 path, bit for bit."""
    els = synth.fcc_sphere(n=300, seed=0)
    els[0][1] = els[0][0] + 1e-3
    q = synth.q_mesh(0.1, 10.0, 1024)
    try:
        I_tc = gpu_ctx.calc_int_debye(els, q, 0, sl=[7.63])
        gpu_ctx.debye_tensor_cores(False)
        I_32 = gpu_ctx.calc_int_debye(els, q, 0, sl=[7.63])
    finally:
        gpu_ctx.debye_tensor_cores(True)
    assert np.array_equal(I_tc, I_32)


def test_coincident_atoms_and_both_paths_agree(gpu_ctx):
    """Coincident atoms add nothing (r = 0 in the reference's sinc is 0); the two paths agree."""
    els = synth.fcc_sphere(n=800, seed=2)
    els = [np.concatenate([els[0], els[0][:5]])]
    q = synth.q_mesh(0.1, 10.0, 1024)
    try:
        I_tc = gpu_ctx.calc_int_debye(els, q, 0, sl=[7.63])
        gpu_ctx.debye_tensor_cores(False)
        I_32 = gpu_ctx.calc_int_debye(els, q, 0, sl=[7.63])
    finally:
        gpu_ctx.debye_tensor_cores(True)
    assert rel_err(I_tc, I_32) < TOL_I


@pytest.mark.parametrize("nshard", [2, 3])
def test_tensor_path_partial_debye_shards(gpu_ctx, nshard):
    """Partial Debye (3 blocks) on the tensor cores: the shards add up to the one-call result."""
    g = load_golden("partial__rocksalt_3blocks")
    els = split_elements(g["xyz"], g["n_el"])
    q = g["q"]
    neb = np.asarray(g["n_el_block"])
    full = gpu_ctx.calc_int_partial_debye(els, neb, q, int(g["source"]), sl=g["sl"])
    parts = sum(shard.int_debye_shard(gpu_ctx, els, q, int(g["source"]), sl=g["sl"], shard=s, nshard=nshard,
                                      n_el_block=neb.ravel()) for s in range(nshard))
    # the cross-block parts cross zero: compare against the total intensity's scale at each q
    scale = np.tile(np.abs(full[:len(q)]), len(full) // len(q))
    assert float(np.max(np.abs(parts - full) / scale)) < 1e-12
