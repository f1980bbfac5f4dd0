"""CPU: the random-circuit generators of the mirror (src/algorithms/rqc.rs:11-232;
the reference's own tests/algorithms/test_rqc.rs is empty).  Checked: names,
one gate type per depth step (1 operation, or 3 for the CZ and SWAP
decompositions), qubits in range, determinism per seed, the weights, the
single-qubit fallback of two-qubit steps on one qubit, invalid weights falling
back to single-qubit gates, and the 2-design's depth 2 n^2."""
import pytest

from logosq_b200 import rqc
from logosq_b200.algorithms import RandomCircuitConfig, RandomGateType

SINGLE = {"H", "X", "Y", "Z", "S", "T"}


def names(c):
    return [op.name() for op in c.operations()]


def steps(c):
    """Split the operation list back into depth steps."""
    ops, out, i = names(c), [], 0
    while i < len(ops):
        if ops[i] == "H" and i + 2 < len(ops) and ops[i + 1].startswith("CNOT") \
                and ops[i + 2] == "H" and c.operations()[i].qubits() == c.operations()[i + 2].qubits():
            out.append("CZ")
            i += 3
        elif ops[i].startswith("CNOT") and i + 2 < len(ops) and ops[i + 1].startswith("CNOT") \
                and ops[i + 2].startswith("CNOT"):
            q = [c.operations()[i + k].qubits() for k in range(3)]
            if q[0] == q[2] and q[1] == q[0][::-1]:
                out.append("SWAP")
                i += 3
                continue
            out.append(ops[i])
            i += 1
        else:
            out.append(ops[i])
            i += 1
    return out


def test_default_config_matches_reference_default():
    cfg = RandomCircuitConfig()
    assert (cfg.num_qubits, cfg.depth, cfg.seed) == (3, 10, None)
    assert cfg.gate_types == [(RandomGateType.Single, 0.5), (RandomGateType.TwoQubit, 0.3),
                              (RandomGateType.Rotation, 0.2)]


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_generate_structure_and_determinism(seed):
    cfg = RandomCircuitConfig(5, 40, seed=seed)
    c = rqc.generate(cfg)
    assert c.name() == "Random Circuit (d=40)" and c.num_qubits() == 5
    assert 40 <= len(c.operations()) <= 120
    assert all(0 <= q < 5 for op in c.operations() for q in op.qubits())
    assert names(c) == names(rqc.generate(RandomCircuitConfig(5, 40, seed=seed)))


def test_rotation_only_weights():
    c = rqc.generate(RandomCircuitConfig(3, 25, [(RandomGateType.Rotation, 1.0)], seed=4))
    assert len(c.operations()) == 25
    assert all(n.startswith(("RX", "RY", "RZ")) for n in names(c))


def test_two_qubit_steps_on_one_qubit_fall_back():
    c = rqc.generate(RandomCircuitConfig(1, 20, [(RandomGateType.TwoQubit, 1.0)], seed=5))
    assert len(c.operations()) == 20 and set(names(c)) <= SINGLE


def test_invalid_weights_give_single_qubit_gates():
    c = rqc.generate(RandomCircuitConfig(3, 15, [(RandomGateType.TwoQubit, -1.0)], seed=6))
    assert len(c.operations()) == 15 and set(names(c)) <= SINGLE


def test_weights_are_respected():
    c = rqc.generate(RandomCircuitConfig(4, 3000, [(RandomGateType.Single, 0.25),
                                                   (RandomGateType.Rotation, 0.75)], seed=7))
    rot = sum(n.startswith(("RX", "RY", "RZ")) for n in names(c)) / 3000
    assert abs(rot - 0.75) < 0.03


def test_generate_simple_and_two_qubit_decompositions():
    c = rqc.generate_simple(4, 400, seed=8)
    assert c.name() == "Random Circuit (d=400)"
    kinds = steps(c)
    assert len(kinds) == 400
    assert {"CZ", "SWAP"} <= set(kinds)


def test_generate_2design():
    c = rqc.generate_2design(3, seed=9)
    assert c.name() == "2-Design Random Circuit (n=3, d=18)"
    assert len(steps(c)) == 18
