"""CPU: the pair formula the Pauli-sum kernels evaluate, restated in numpy and
checked against the oracle (PauliTerm::expectation,
src/optimization/observable.rs:95-147).

Terms sharing an X mask x are summed over pairs (i, j = i ^ x), i with the top
bit of x clear.  With W = conj(a_i) a_j = wr + i wi and, per term, the sign
s(i) = (-1)^popcount(i & z) and selectors (ca, cb) of the Y phase, the pair
contributes wr (A_i + A_j) + wi (B_i - B_j), A = sum s ca, B = sum s cb.  Since
s(j) = s(i) (-1)^ny and ca = 0 for odd ny, cb = 0 for even ny, A_j = A_i and
B_j = -B_i: the kernels evaluate 2 (wr A_i + wi B_i)."""
import numpy as np
import pytest

import oracle
from logosq_b200 import abi, workloads


def selectors(ny, textbook):
    k = ny & 3
    if textbook:
        k = (4 - k) & 3
    return ({0: 1.0, 2: -1.0}.get(k, 0.0), {1: -1.0, 3: 1.0}.get(k, 0.0))


def pair_formula(v, terms, textbook):
    n = int(np.log2(len(v)))
    idx = np.arange(len(v), dtype=np.uint64)
    total = 0.0
    for x in sorted({int(t) for t in terms["xmask"]}):
        grp = terms[terms["xmask"] == x]
        ca = np.array([c * selectors(int(ny), textbook)[0] for c, ny in zip(grp["coefficient"], grp["ny"])])
        cb = np.array([c * selectors(int(ny), textbook)[1] for c, ny in zip(grp["coefficient"], grp["ny"])])

        def sums(i):
            par = np.array([[bin(int(k) & int(z)).count("1") & 1 for z in grp["zmask"]] for k in i])
            s = 1.0 - 2.0 * par
            return s @ ca, s @ cb

        if x == 0:
            a_sum, _ = sums(idx)
            total += float(np.sum(np.abs(v) ** 2 * a_sum))
            continue
        hb = x.bit_length() - 1
        i = idx[(idx >> np.uint64(hb)) & np.uint64(1) == 0]
        j = i ^ np.uint64(x)
        w = np.conj(v[i]) * v[j]
        ai, bi = sums(i)
        aj, bj = sums(j)
        np.testing.assert_array_equal(aj, ai)
        np.testing.assert_array_equal(bj, -bi)
        total += float(np.sum(2.0 * (w.real * ai + w.imag * bi)))
    assert n > 0
    return total


def random_terms(n, count, seed):
    rng = workloads.SplitMix64(seed)
    terms = np.zeros(count, dtype=abi.TERM_DTYPE)
    for t in range(count):
        x = rng.randint(0, (1 << n) - 1) if t % 4 else 0
        if t % 5 == 1:
            x = terms[t - 1]["xmask"]  # shared X masks: several terms per group
        z = rng.randint(0, (1 << n) - 1)
        terms[t]["coefficient"] = rng.uniform(-1, 1)
        terms[t]["xmask"] = x
        terms[t]["zmask"] = z
        terms[t]["ny"] = bin(int(x) & z).count("1")
    return terms


@pytest.mark.parametrize("textbook", [False, True])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_pair_formula_matches_oracle(seed, textbook):
    n = 7
    v = workloads.gaussian_state(n, seed)
    terms = random_terms(n, 24, seed)
    yc = abi.Y_TEXTBOOK if textbook else abi.Y_REFERENCE
    want = oracle.expectation(v, terms, yc)
    got = pair_formula(v, terms, textbook)
    assert abs(got - want) < 1e-12 * max(1.0, abs(want))


def test_pair_formula_on_xyz_chain():
    n = 8
    c = workloads.uniform_stream(9, 3 * (n - 1) + 1, -1.0, 1.0)
    terms = workloads.heisenberg_terms(n, c[:n - 1], c[n - 1:2 * (n - 1)], c[2 * (n - 1):3 * (n - 1)],
                                       0.5 * c[-1])
    v = workloads.gaussian_state(n, 4)
    want = oracle.expectation(v, terms, abi.Y_REFERENCE)
    assert abs(pair_formula(v, terms, False) - want) < 1e-12 * max(1.0, abs(want))


def zfold_formula(v, terms):
    """The folded form of the X-mask-0 group (k_pauli_zfold), vectorised over the
    256 threads: per 4096-amplitude chunk and thread, the terms' signs at the
    bits the thread keeps fixed are folded into 16 coefficients by bits 8-11 of
    z, and a Walsh-Hadamard transform gives the signed sum for each k."""
    n = int(np.log2(len(v)))
    pr = np.abs(v) ** 2
    z = terms["zmask"].astype(np.int64)
    ca = terms["coefficient"].astype(np.float64)  # X mask 0: the real selector is 1
    pat = (z >> 8) & 15
    tid = np.arange(256, dtype=np.int64)
    total = 0.0
    for c in range(1 << (n - 12)):
        fixed = (c << 12) | tid
        C = np.zeros((16, 256))
        for t in range(len(z)):
            par = np.array([bin(int(f) & int(z[t])).count("1") & 1 for f in fixed])
            C[pat[t]] += np.where(par == 1, -ca[t], ca[t])
        hs = 1
        while hs < 16:
            for q in range(16):
                if not q & hs:
                    C[q], C[q | hs] = C[q] + C[q | hs], C[q] - C[q | hs]
            hs <<= 1
        for k in range(16):
            total += float(np.sum(pr[fixed | (k << 8)] * C[k]))
    return total


def test_zfold_formula_matches_oracle():
    n = 13
    rng = workloads.SplitMix64(17)
    terms = np.zeros(30, dtype=abi.TERM_DTYPE)
    for t in range(30):
        terms[t]["coefficient"] = rng.uniform(-1, 1)
        terms[t]["zmask"] = rng.randint(0, (1 << n) - 1)
    v = workloads.gaussian_state(n, 8)
    want = oracle.expectation(v, terms, abi.Y_REFERENCE)
    assert abs(zfold_formula(v, terms) - want) < 1e-12 * max(1.0, abs(want))
