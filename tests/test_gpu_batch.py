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


def _make(recs, share, templates=None, extra_params=0):
    import os
    from logosq_b200.batch import BatchedParameterShift
    old = os.environ.get("LQ_BATCH_PREFIX")
    os.environ["LQ_BATCH_PREFIX"] = "1" if share else "0"
    try:
        specs = []
        for k, r in enumerate(recs):
            n = r["n"]
            g = templates[k] if templates else workloads.basic_entangling_template(n, 4)
            specs.append((n, g, 8 * n + extra_params,
                          workloads.heisenberg_terms(n, r["jx"], r["jy"], r["jz"], r["h"])))
        return BatchedParameterShift(specs)
    finally:
        if old is None:
            del os.environ["LQ_BATCH_PREFIX"]
        else:
            os.environ["LQ_BATCH_PREFIX"] = old


@pytest.mark.parametrize("tile_bits", [10, 11, 12])
def test_shared_prefixes_are_bitwise_the_unshared_launch(tile_bits):
    """Shifted circuits that start from the base circuit's checkpoints give
    exactly the energies of circuits run from |0...0> (same sums, same order),
    for states in shared memory (n <= 12) and in HBM slots (n > 12)."""
    recs = workloads.heisenberg_instances(10, seed=31, n_lo=9, n_hi=15)
    theta = np.concatenate([r["theta"] for r in recs])
    out = {}
    for share in (True, False):
        b = _make(recs, share)
        call("lq_batch_set_tile_bits", b._h, tile_bits)
        info = b.tuning()
        assert info["shared_prefixes"] == share
        assert (info["checkpoint_bytes"] > 0) == share
        out[share] = b.gradients(theta)
        e2, g2 = b.gradients(theta + 0.05)  # the graph replays with new angles
        out[(share, 1)] = (e2, g2)
    assert np.array_equal(out[True][0], out[False][0])
    assert np.array_equal(out[True][1], out[False][1])
    assert np.array_equal(out[(True, 1)][1], out[(False, 1)][1])
    # and the plain path agrees
    gs = np.split(out[True][1], np.cumsum([8 * r["n"] for r in recs])[:-1])
    for i in (0, len(recs) - 1):
        r = recs[i]
        n = r["n"]
        _, g_plain = plain_gradient(n, workloads.basic_entangling_template(n, 4), r["theta"],
                                    workloads.heisenberg_terms(n, r["jx"], r["jy"], r["jz"],
                                                               r["h"]))
        assert np.abs(gs[i] - g_plain).max() < 1e-10


def test_shared_prefixes_with_reused_and_unused_parameters():
    """A parameter bound to gates in two layers starts at its first gate; a
    parameter bound to none keeps a zero gradient."""
    recs = workloads.heisenberg_instances(3, seed=41, n_lo=11, n_hi=14)
    temps = []
    for r in recs:
        g = workloads.basic_entangling_template(r["n"], 4).copy()
        ry = np.nonzero(g["kind"] == abi.RY)[0]
        g["param"][ry[-1], 0] = g["param"][ry[0], 0]  # last RY reuses parameter 0
        temps.append(g)
    P = [8 * r["n"] + 1 for r in recs]
    rng = np.random.default_rng(3)
    theta = rng.uniform(-np.pi, np.pi, sum(P))
    res = {s: _make(recs, s, temps, extra_params=1).gradients(theta) for s in (True, False)}
    assert np.array_equal(res[True][1], res[False][1])
    gs = np.split(res[True][1], np.cumsum(P)[:-1])
    off = 0
    for i, r in enumerate(recs):
        n = r["n"]
        th = theta[off:off + P[i]]
        off += P[i]
        g_or = oracle.parameter_shift(n, temps[i], th, workloads.heisenberg_terms(
            n, r["jx"], r["jy"], r["jz"], r["h"]))
        assert np.abs(gs[i] - g_or).max() < 1e-10
        assert gs[i][-1] == 0.0


def _random_observable(n, rng):
    """Pauli sum with several terms per X mask (odd and even Y counts, Z bits
    anywhere) and a Z-only group with Z masks over all index bits."""
    rows = []
    for _ in range(4):
        w = int(rng.integers(1, 4))
        lo = int(rng.integers(0, n - w + 1))
        x = sum(1 << (lo + k) for k in range(w))
        for _ in range(int(rng.integers(1, 5))):
            z = int(rng.integers(0, 1 << n))
            rows.append((float(rng.normal()), x, z, bin(x & z).count("1")))
    for _ in range(24):
        z = int(rng.integers(1, 1 << n))
        rows.append((float(rng.normal()), 0, z, 0))
    arr = np.zeros(len(rows), dtype=abi.TERM_DTYPE)
    for k, (c, x, z, ny) in enumerate(rows):
        arr[k]["coefficient"] = c
        arr[k]["xmask"] = np.uint64(x)
        arr[k]["zmask"] = np.uint64(z)
        arr[k]["ny"] = ny
    return arr


@pytest.mark.parametrize("tile_bits", [10, 12])
def test_batch_general_observables_match_plain(tile_bits):
    """Energy windows with more than two terms per X mask, odd Y counts and a
    folded Z-only group whose terms spread over every tile bit."""
    from logosq_b200.batch import BatchedParameterShift
    rng = np.random.default_rng(17)
    specs, thetas = [], []
    for n in (7, 11, 13, 15):
        gates = workloads.basic_entangling_template(n, 2)
        terms = _random_observable(n, rng)
        specs.append((n, gates, 4 * n, terms))
        thetas.append(rng.uniform(-np.pi, np.pi, 4 * n))
    b = BatchedParameterShift(specs)
    call("lq_batch_set_tile_bits", b._h, tile_bits)
    e, g = b.gradients(np.concatenate(thetas))
    gs = b.split(g)
    for i, (n, gates, _, terms) in enumerate(specs):
        e_plain, g_plain = plain_gradient(n, gates, thetas[i], terms)
        assert abs(e[i] - e_plain) < 1e-12 * max(1, abs(e_plain)), (n, e[i], e_plain)
        assert np.abs(gs[i] - g_plain).max() < 1e-10, n
