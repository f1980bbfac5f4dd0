"""GPU: the batched parameter-shift engine against the plain per-circuit path
(lq_parameter_shift) and the CPU oracle.  Gradients must match to 1e-10."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from logosq_b200 import State, abi, workloads
from logosq_b200._lib import call
from logosq_b200.batch import heisenberg_batch

pytestmark = pytest.mark.gpu


def plain_gradient(n, gates, theta, terms):
    st = State.zero_state(n)
    g = np.zeros(len(theta))
    call("lq_parameter_shift", st.handle, abi.gate_ptr(gates), len(gates), abi.f64_ptr(theta),
         len(theta), abi.term_ptr(terms), len(terms), abi.Y_REFERENCE, math.pi / 2,
         abi.f64_ptr(g))
    e = C.c_double()
    call("lq_ansatz_energy", st.handle, abi.gate_ptr(gates), len(gates), abi.f64_ptr(theta),
         len(theta), abi.term_ptr(terms), len(terms), abi.Y_REFERENCE, C.byref(e))
    return e.value, g


def test_batch_matches_plain_and_oracle_small():
    recs = workloads.heisenberg_instances(6, seed=4, n_lo=6, n_hi=11)
    b = heisenberg_batch(recs)
    theta = np.concatenate([r["theta"] for r in recs])
    e, g = b.gradients(theta)
    gs = b.split(g)
    for i, r in enumerate(recs):
        n = r["n"]
        gates = workloads.basic_entangling_template(n, 4)
        terms = workloads.heisenberg_terms(n, r["jx"], r["jy"], r["jz"], r["h"])
        e_plain, g_plain = plain_gradient(n, gates, r["theta"], terms)
        assert abs(e[i] - e_plain) < 1e-12 * max(1, abs(e_plain))
        assert np.abs(gs[i] - g_plain).max() < 1e-10
        g_or = oracle.parameter_shift(n, gates, r["theta"], terms)
        assert np.abs(gs[i] - g_or).max() < 1e-10


@pytest.mark.parametrize("n", [13, 15])
def test_batch_tiled_instances_match_plain(n):
    """n > 12: states in HBM slots swept by tiles; every autotuner candidate."""
    recs = [r for r in workloads.heisenberg_instances(40, seed=7, n_lo=n, n_hi=n)][:2]
    b = heisenberg_batch(recs)
    theta = np.concatenate([r["theta"] for r in recs])
    e, g = b.gradients(theta)
    e2, g2 = b.gradients(theta)  # second call replays the captured graph
    assert np.array_equal(g, g2) and np.array_equal(e, e2)
    gs = b.split(g)
    for i, r in enumerate(recs):
        gates = workloads.basic_entangling_template(n, 4)
        terms = workloads.heisenberg_terms(n, r["jx"], r["jy"], r["jz"], r["h"])
        e_plain, g_plain = plain_gradient(n, gates, r["theta"], terms)
        assert abs(e[i] - e_plain) < 1e-12 * max(1, abs(e_plain))
        assert np.abs(gs[i] - g_plain).max() < 1e-10
    assert b.tuning()["tile_bits"] in (10, 11, 12)


def test_batch_mixed_sizes_and_new_theta():
    recs = workloads.heisenberg_instances(12, seed=11, n_lo=8, n_hi=14)
    b = heisenberg_batch(recs)
    theta = np.concatenate([r["theta"] for r in recs])
    b.gradients(theta)
    theta2 = theta + 0.1
    e, g = b.gradients(theta2)
    gs = b.split(g)
    for i, r in enumerate(recs):
        n = r["n"]
        gates = workloads.basic_entangling_template(n, 4)
        terms = workloads.heisenberg_terms(n, r["jx"], r["jy"], r["jz"], r["h"])
        _, g_plain = plain_gradient(n, gates, r["theta"] + 0.1, terms)
        assert np.abs(gs[i] - g_plain).max() < 1e-10


@pytest.mark.parametrize("tile_bits", [10, 11, 12])
def test_batch_every_tile_width_matches_plain(tile_bits):
    """Each fusion width the autotuner may pick gives the plain path's gradients
    (at widths below 12 only part of the CTA's threads own amplitudes)."""
    recs = workloads.heisenberg_instances(3, seed=21, n_lo=13, n_hi=15)
    b = heisenberg_batch(recs)
    call("lq_batch_set_tile_bits", b._h, tile_bits)
    theta = np.concatenate([r["theta"] for r in recs])
    e, g = b.gradients(theta)
    assert b.tuning()["tile_bits"] == tile_bits
    gs = b.split(g)
    for i, r in enumerate(recs):
        n = r["n"]
        gates = workloads.basic_entangling_template(n, 4)
        terms = workloads.heisenberg_terms(n, r["jx"], r["jy"], r["jz"], r["h"])
        e_plain, g_plain = plain_gradient(n, gates, r["theta"], terms)
        assert abs(e[i] - e_plain) < 1e-12 * max(1, abs(e_plain))
        assert np.abs(gs[i] - g_plain).max() < 1e-10


def test_batch_set_tile_bits_rejects_unknown_width():
    from logosq_b200 import LogosQError
    b = heisenberg_batch(workloads.heisenberg_instances(1, seed=2, n_lo=13, n_hi=13))
    with pytest.raises(LogosQError) as e:
        call("lq_batch_set_tile_bits", b._h, 9)
    assert e.value.code == abi.LQ_ERR_INVALID_ARG
    call("lq_batch_set_tile_bits", b._h, 0)  # back to autotuning
