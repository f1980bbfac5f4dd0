"""Writes tests/golden/known_answers.json: the known-answer assertions of the
reference's own tests for the dense path, transcribed case by case.

Each case names the reference test it comes from (file:line), the circuit as a
list of builder calls (Circuit::x / h / ... are the dense matrix builders that
renormalise; cnot / swap / toffoli / rx / ... are the gate structs), and the
assertions with the reference's tolerance.  Run:
    python tests/golden/make_known_answers.py
"""
import json
import math
from pathlib import Path

PI = math.pi
R2 = 1.0 / math.sqrt(2.0)

CASES = [
    # ---- tests/test_circuits_dense.rs -------------------------------------
    dict(name="cnot_basic", src="tests/test_circuits_dense.rs:213-238", n=3,
         ops=[["x", 0], ["cnot", 0, 2]],
         checks=[["prob_gt", 5, 0.99]] + [["prob_lt", i, 1e-10] for i in (0, 1, 2, 3, 4, 6, 7)]),
    dict(name="cnot_control_zero", src="tests/test_circuits_dense.rs:239-249", n=3,
         ops=[["x", 0], ["cnot", 0, 2], ["x", 0], ["cnot", 0, 2]],
         checks=[["prob_gt", 1, 0.99]]),
    dict(name="cnot_order_01", src="tests/test_circuits_dense.rs:252-264", n=2,
         ops=[["x", 0], ["cnot", 0, 1]], checks=[["prob_gt", 3, 0.99]]),
    dict(name="cnot_order_10", src="tests/test_circuits_dense.rs:266-276", n=2,
         ops=[["x", 0], ["cnot", 1, 0]], checks=[["prob_gt", 2, 0.99]]),
    dict(name="cnot_distant", src="tests/test_circuits_dense.rs:279-304", n=5,
         ops=[["x", 0], ["cnot", 0, 4]],
         checks=[["prob_gt", 17, 0.99]] + [["prob_lt", i, 1e-10] for i in range(32) if i != 17]),
    dict(name="cnot_chain", src="tests/test_circuits_dense.rs:306-335", n=4,
         ops=[["h", 0], ["cnot", 0, 1], ["cnot", 1, 2], ["cnot", 2, 3]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 15, 0.5, 1e-10]]
         + [["prob_lt", i, 1e-10] for i in range(1, 15)]),
    dict(name="swap_basic", src="tests/test_circuits_dense.rs:339-362", n=3,
         ops=[["x", 0], ["swap", 0, 2]],
         checks=[["prob_gt", 1, 0.99]] + [["prob_lt", i, 1e-10] for i in (0, 2, 3, 4, 5, 6, 7)]),
    dict(name="swap_self_inverse", src="tests/test_circuits_dense.rs:364-373", n=3,
         ops=[["x", 0], ["swap", 0, 2], ["swap", 0, 2]], checks=[["prob_gt", 4, 0.99]]),
    dict(name="multiple_swaps", src="tests/test_circuits_dense.rs:376-408", n=4,
         ops=[["x", 0], ["x", 2], ["swap", 0, 1], ["swap", 2, 3], ["swap", 1, 2]],
         checks=[["prob_gt", 3, 0.99]] + [["prob_lt", i, 1e-10] for i in range(16) if i != 3]),
    dict(name="swap_entangled", src="tests/test_circuits_dense.rs:410-437", n=3,
         ops=[["h", 0], ["cnot", 0, 1], ["swap", 1, 2]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 5, 0.5, 1e-10]]
         + [["prob_lt", i, 1e-10] for i in (1, 2, 3, 4, 6, 7)]),
    dict(name="toffoli_basic", src="tests/test_circuits_dense.rs:442-465", n=3,
         ops=[["x", 0], ["x", 1], ["toffoli", 0, 1, 2]],
         checks=[["prob_gt", 7, 0.99]] + [["prob_lt", i, 1e-10] for i in range(7)]),
    dict(name="toffoli_one_control", src="tests/test_circuits_dense.rs:467-476", n=3,
         ops=[["x", 0], ["toffoli", 0, 1, 2]], checks=[["prob_gt", 4, 0.99]]),
    dict(name="toffoli_control_order", src="tests/test_circuits_dense.rs:479-504", n=3,
         ops=[["x", 0], ["x", 1], ["toffoli", 1, 0, 2]], checks=[["prob_gt", 7, 0.99]]),
    dict(name="toffoli_distant", src="tests/test_circuits_dense.rs:506-545", n=5,
         ops=[["x", 0], ["x", 4], ["toffoli", 0, 4, 2]],
         checks=[["prob_gt", 21, 0.99]] + [["prob_lt", i, 1e-10] for i in range(32) if i != 21]),
    dict(name="toffoli_superposition", src="tests/test_circuits_dense.rs:547-577", n=3,
         ops=[["h", 0], ["x", 1], ["toffoli", 0, 1, 2]],
         checks=[["prob_eq", 2, 0.5, 1e-10], ["prob_eq", 7, 0.5, 1e-10]]
         + [["prob_lt", i, 1e-10] for i in (0, 1, 3, 4, 5, 6)]),
    dict(name="toffoli_chain", src="tests/test_circuits_dense.rs:579-607", n=5,
         ops=[["x", 0], ["x", 1], ["x", 2], ["toffoli", 0, 1, 3], ["toffoli", 2, 3, 4]],
         checks=[["prob_gt", 31, 0.99]]),
    dict(name="toffoli_self_inverse", src="tests/test_circuits_dense.rs:609-627", n=3,
         ops=[["x", 0], ["x", 1], ["toffoli", 0, 1, 2], ["toffoli", 0, 1, 2]],
         checks=[["prob_gt", 6, 0.99]]),
    dict(name="bell", src="tests/test_circuits_dense.rs:631-646", n=2,
         ops=[["h", 0], ["cnot", 0, 1]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_lt", 1, 1e-10], ["prob_lt", 2, 1e-10],
                 ["prob_eq", 3, 0.5, 1e-10]]),
    dict(name="bell_flipped", src="tests/test_circuits_dense.rs:648-666", n=2,
         ops=[["x", 0], ["h", 0], ["cnot", 0, 1]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_lt", 1, 1e-10], ["prob_lt", 2, 1e-10],
                 ["prob_eq", 3, 0.5, 1e-10]]),
    dict(name="ghz_dense_matrices", src="tests/test_circuits_dense.rs:668-727", n=3,
         ops=[["h", 0],
              ["dense", [[0, 0], [1, 1], [2, 2], [3, 3], [4, 6], [5, 7], [6, 4], [7, 5]]],
              ["dense", [[0, 0], [1, 1], [4, 4], [5, 5], [2, 3], [3, 2], [6, 7], [7, 6]]]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 7, 0.5, 1e-10]]
         + [["prob_lt", i, 1e-10] for i in range(1, 7)]),
    dict(name="ghz_simple", src="tests/test_circuits_dense.rs:729-749", n=3,
         ops=[["h", 0], ["cnot", 0, 1], ["cnot", 0, 2]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 7, 0.5, 1e-10]]
         + [["prob_lt", i, 1e-10] for i in range(1, 7)]),
    dict(name="cnot_preexisting_entanglement", src="tests/test_circuits_dense.rs:751-777", n=3,
         ops=[["h", 0], ["cnot", 0, 1], ["cnot", 1, 2]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 7, 0.5, 1e-10]]
         + [["prob_lt", i, 1e-10] for i in range(1, 7)]),
    dict(name="expectation_x_plus", src="tests/test_circuits_dense.rs:779-798", n=1,
         ops=[["h", 0]],
         checks=[["expect_matrix", [[0, 0], [1, 0], [1, 0], [0, 0]], 1.0, 1e-10],
                 ["expect_matrix", [[1, 0], [0, 0], [0, 0], [-1, 0]], 0.0, 1e-10]]),
    # ---- tests/test_gates_parameterized.rs --------------------------------
    dict(name="rx_pi", src="tests/test_gates_parameterized.rs:14-28", n=1, ops=[["rx", 0, PI]],
         checks=[["abs_lt", 0, 1e-10], ["abs_eq", 1, 1.0, 1e-10], ["arg_eq", 1, -PI / 2, 1e-10]]),
    dict(name="rx_half_pi", src="tests/test_gates_parameterized.rs:31-43", n=1,
         ops=[["rx", 0, PI / 2]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 1, 0.5, 1e-10]]),
    dict(name="ry_pi", src="tests/test_gates_parameterized.rs:45-56", n=1, ops=[["ry", 0, PI]],
         checks=[["abs_lt", 0, 1e-10], ["amp_eq", 1, [1.0, 0.0], 1e-10]]),
    dict(name="ry_half_pi", src="tests/test_gates_parameterized.rs:58-76", n=1,
         ops=[["ry", 0, PI / 2]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 1, 0.5, 1e-10], ["imag_lt", 0, 1e-10],
                 ["imag_lt", 1, 1e-10]]),
    dict(name="rz_pi_then_h", src="tests/test_gates_parameterized.rs:78-98", n=1,
         ops=[["h", 0], ["rz", 0, PI], ["h", 0]],
         checks=[["prob_lt", 0, 1e-10], ["prob_eq", 1, 1.0, 1e-10]]),
    dict(name="rz_preserves_probabilities", src="tests/test_gates_parameterized.rs:100-118", n=1,
         ops=[["h", 0], ["rz", 0, PI / 4]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 1, 0.5, 1e-10]]),
    dict(name="phase_gate", src="tests/test_gates_parameterized.rs:120-135", n=1,
         ops=[["h", 0], ["phase", 0, PI / 2]],
         checks=[["amp_eq", 0, [R2, 0.0], 1e-10], ["amp_eq", 1, [0.0, R2], 1e-10]]),
    dict(name="u3_as_x", src="tests/test_gates_parameterized.rs:137-149", n=1,
         ops=[["u3", 0, PI, 0.0, PI]],
         checks=[["prob_lt", 0, 1e-10], ["prob_eq", 1, 1.0, 1e-10]]),
    dict(name="u3_as_h", src="tests/test_gates_parameterized.rs:151-163", n=1,
         ops=[["u3", 0, PI / 2, 0.0, PI]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_eq", 1, 0.5, 1e-10]]),
    dict(name="crx_control_zero", src="tests/test_gates_parameterized.rs:170-181", n=2,
         ops=[["crx", 0, 1, PI]], checks=[["prob_eq", 0, 1.0, 1e-10]]),
    dict(name="crx_control_one", src="tests/test_gates_parameterized.rs:183-195", n=2,
         ops=[["x", 0], ["crx", 0, 1, PI]],
         checks=[["prob_lt", 0, 1e-10], ["prob_lt", 1, 1e-10], ["prob_lt", 2, 1e-10],
                 ["prob_eq", 3, 1.0, 1e-10]]),
    dict(name="cry", src="tests/test_gates_parameterized.rs:198-213", n=2,
         ops=[["x", 0], ["cry", 0, 1, PI / 2]],
         checks=[["prob_eq", 2, 0.5, 1e-10], ["prob_eq", 3, 0.5, 1e-10]]),
    dict(name="crz", src="tests/test_gates_parameterized.rs:215-238", n=2,
         ops=[["x", 0], ["h", 1], ["crz", 0, 1, PI]],
         checks=[["prob_eq", 2, 0.5, 1e-10], ["prob_eq", 3, 0.5, 1e-10],
                 ["absarg_ratio_eq", 3, 2, PI, 1e-10]]),
    dict(name="cphase_param", src="tests/test_gates_parameterized.rs:240-262", n=2,
         ops=[["h", 0], ["h", 1], ["cphase_param", 0, 1, PI / 2]],
         checks=[["prob_eq", i, 0.25, 1e-10] for i in range(4)]),
    dict(name="rxx_entangles", src="tests/test_gates_parameterized.rs:269-284", n=2,
         ops=[["h", 0], ["rxx", 0, 1, PI / 2]], checks=[["nonzero_count_gt", 1e-10, 1]]),
    dict(name="ryy_probabilities", src="tests/test_gates_parameterized.rs:286-302", n=2,
         ops=[["h", 0], ["h", 1], ["ryy", 0, 1, PI / 4]],
         checks=[["prob_eq", i, 0.25, 1e-10] for i in range(4)]),
    dict(name="rzz_probabilities", src="tests/test_gates_parameterized.rs:304-320", n=2,
         ops=[["h", 0], ["h", 1], ["rzz", 0, 1, PI / 4]],
         checks=[["prob_eq", i, 0.25, 1e-10] for i in range(4)]),
    dict(name="rzz_phase", src="tests/test_gates_parameterized.rs:322-335", n=2,
         ops=[["rzz", 0, 1, PI]], checks=[["amp_eq", 0, [0.0, -1.0], 1e-10]]),
    dict(name="vqc_pattern_normalised", src="tests/test_gates_parameterized.rs:342-361", n=2,
         ops=[["ry", 0, 0.5], ["ry", 1, 0.3], ["rzz", 0, 1, 0.7], ["ry", 0, 0.2], ["ry", 1, 0.4]],
         checks=[["norm_eq", 1.0, 1e-10]]),
    dict(name="rotation_composition", src="tests/test_gates_parameterized.rs:387-413", n=1,
         ops=[["h", 0], ["rz", 0, 0.3], ["rz", 0, 0.7]],
         checks=[["same_as", [["h", 0], ["rz", 0, 1.0]], 1e-10]]),
    dict(name="zero_angle_identity", src="tests/test_gates_parameterized.rs:416-428", n=1,
         ops=[["ry", 0, 0.0]], checks=[["prob_eq", 0, 1.0, 1e-10], ["prob_lt", 1, 1e-10]]),
    dict(name="bell_parameterized", src="tests/test_gates_parameterized.rs:430-446", n=2,
         ops=[["ry", 0, PI / 2], ["rz", 0, PI], ["cnot", 0, 1]],
         checks=[["prob_eq", 0, 0.5, 1e-10], ["prob_lt", 1, 1e-10], ["prob_lt", 2, 1e-10],
                 ["prob_eq", 3, 0.5, 1e-10]]),
    dict(name="multiple_rzz", src="tests/test_gates_parameterized.rs:452-479", n=2,
         ops=[["h", 0], ["h", 1]] + [["rzz", 0, 1, PI / 8]] * 4,
         checks=[["same_as", [["h", 0], ["h", 1], ["rzz", 0, 1, PI / 2]], 1e-10]]),
    dict(name="large_angle_wrap", src="tests/test_gates_parameterized.rs:481-497", n=1,
         ops=[["ry", 0, 2 * PI]], checks=[["prob_eq", 0, 1.0, 1e-10], ["prob_lt", 1, 1e-10]]),
    # ---- tests/test_qft.rs (qft::apply equals the gate QFT) ---------------
    dict(name="qft_basis_one", src="tests/test_qft.rs:58-76", n=1,
         ops=[["x", 0], ["qft"]],
         checks=[["amp_eq", 0, [R2, 0.0], 1e-5], ["amp_eq", 1, [-R2, 0.0], 1e-5]]),
    dict(name="qft_known_transformation", src="tests/test_qft.rs:130-147", n=1,
         ops=[["h", 0], ["qft"]], checks=[["abs_eq", 0, 1.0, 1e-5], ["abs_lt", 1, 1e-5]]),
    dict(name="qft_multi_qubit", src="tests/test_qft.rs:149-168", n=2,
         ops=[["h", 0], ["h", 1], ["qft"]],
         checks=[["abs_eq", 0, 1.0, 1e-5]] + [["abs_lt", i, 1e-5] for i in (1, 2, 3)]),
    dict(name="qft_correctness_001", src="tests/test_qft.rs:190-224", n=3,
         ops=[["x", 2], ["qft"]],
         checks=[["abs_eq", i, 1 / math.sqrt(8), 1e-5] for i in range(8)]
         + [["phase_mod_eq", i, 2 * PI * i / 8, 1e-5] for i in range(8)]),
    dict(name="qft_inverse_identity_4", src="tests/test_qft.rs:78-128", n=4,
         ops=[["h", 0], ["x", 1], ["h", 2], ["x", 3], ["qft"], ["iqft"]],
         checks=[["same_as", [["h", 0], ["x", 1], ["h", 2], ["x", 3]], 1e-5]]),
]
for n in range(1, 11):  # tests/test_qft.rs:226-281
    chk = [["abs_eq", i, 1 / math.sqrt(2 ** n), 1e-5] for i in range(min(2 ** n, 64))]
    if n <= 6:
        chk += [["imag_lt", i, 1e-5] for i in range(2 ** n)] + [["real_gt", i, 0.0]
                                                               for i in range(2 ** n)]
    CASES.append(dict(name=f"qft_zero_state_{n}", src="tests/test_qft.rs:226-281", n=n,
                      ops=[["qft"]], checks=chk))

# Observables: tests/test_optimization_observables.rs (state prep, terms, value).
OBSERVABLES = [
    dict(name="z_on_zero", src="tests/test_optimization_observables.rs:32-41", n=1, ops=[],
         terms=[[1.0, "Z"]], value=1.0),
    dict(name="z_on_one", src="tests/test_optimization_observables.rs:43-57", n=1, ops=[["x", 0]],
         terms=[[1.0, "Z"]], value=-1.0),
    dict(name="x_on_plus", src="tests/test_optimization_observables.rs:59-73", n=1,
         ops=[["h", 0]], terms=[[1.0, "X"]], value=1.0),
    dict(name="single_z_2", src="tests/test_optimization_observables.rs:75-82", n=2, ops=[],
         terms=[[1.0, "ZI"]], value=1.0),
    dict(name="zz_00", src="tests/test_optimization_observables.rs:84-111", n=2, ops=[],
         terms=[[1.0, "ZZ"]], value=1.0),
    dict(name="zz_11", src="tests/test_optimization_observables.rs:84-111", n=2,
         ops=[["x", 0], ["x", 1]], terms=[[1.0, "ZZ"]], value=1.0),
    dict(name="zz_01", src="tests/test_optimization_observables.rs:84-111", n=2, ops=[["x", 1]],
         terms=[[1.0, "ZZ"]], value=-1.0),
    dict(name="ising_00", src="tests/test_optimization_observables.rs:113-124", n=2, ops=[],
         terms=[[1.0, "ZZ"], [0.5, "ZI"], [0.5, "IZ"]], value=2.0),
    dict(name="z0_plus_z1", src="tests/test_optimization_observables.rs:126-139", n=2, ops=[],
         terms=[[1.0, "ZI"], [1.0, "IZ"]], value=2.0),
]

# State-level: tests/test_normalize.rs, tests/test_parallel.rs.
STATES = [
    dict(name="normalize_vector", src="tests/test_normalize.rs:14-40",
         vector=[[2.0, 1.0], [1.0, 3.0], [-1.0, 2.0], [0.5, -0.5]], tol=1e-10),
    dict(name="normalize_zero_vector", src="tests/test_normalize.rs:58-68",
         vector=[[0, 0], [0, 0], [0, 0], [0, 0]], tol=1e-10),
]
INNER = [
    dict(name="zero_one", src="tests/test_parallel.rs:82-88", a="zero2", b="one2", value=[0, 0]),
    dict(name="zero_zero", src="tests/test_parallel.rs:90-95", a="zero2", b="zero2",
         value=[1, 0]),
    dict(name="zero_plus", src="tests/test_parallel.rs:97-102", a="zero2", b="plus2",
         value=[0.5, 0]),
    dict(name="zero_bell", src="tests/test_parallel.rs:104-109", a="zero2", b="bell",
         value=[R2, 0]),
    dict(name="custom", src="tests/test_parallel.rs:111-140",
         a=[[0.5, 0], [0, 0.5], [-0.5, 0], [0, -0.5]], b=[[0.5, 0], [0.5, 0], [0.5, 0], [0.5, 0]],
         value="manual"),
]

if __name__ == "__main__":
    out = Path(__file__).with_name("known_answers.json")
    out.write_text(json.dumps({"circuits": CASES, "observables": OBSERVABLES, "states": STATES,
                               "inner_products": INNER}, indent=1))
    print(f"wrote {out} ({len(CASES)} circuit cases)")
