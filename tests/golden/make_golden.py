"""Extract the reference's own known-answer fixtures into ``tests/golden/reference_fixtures.json``.

The reference's hot-path tests cannot run here (they need JAX and the empty
``general_python`` submodule), so their fixtures are read from the test
sources as text: the literal arrays are taken from the syntax tree of each
file and the expected values from the literals in their asserts.  Run from
the repository root with the reference checked out at ``--ref``:

    python tests/golden/make_golden.py --ref /root/reference

Only the fixture values are stored; the tests in ``tests/`` recompute every
expected value with the oracle and compare.
"""

from __future__ import annotations

import argparse
import ast
import json
import os


def _load(path):
    with open(path, "r", encoding="utf-8") as fh:
        return ast.parse(fh.read(), filename=path)


def _func(tree, name):
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == name:
            return node
    raise KeyError(name)


def _first_array_literal(fn):
    for node in ast.walk(fn):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", None) in ("array", "asarray") and node.args:
            try:
                return ast.literal_eval(node.args[0])
            except ValueError:
                continue
    raise ValueError(f"no literal array in {fn.name}")


def _assign_literal(fn, target):
    for node in ast.walk(fn):
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == target for t in node.targets):
            v = node.value
            if isinstance(v, ast.Call) and v.args:
                return ast.literal_eval(v.args[0])
            return ast.literal_eval(v)
    raise KeyError(target)


def _cplx(x):
    if isinstance(x, list):
        return [_cplx(v) for v in x]
    c = complex(x)
    return [c.real, c.imag]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "reference_fixtures.json"))
    args = ap.parse_args()
    tests = os.path.join(args.ref, "Python", "tests")
    out = {}

    # (1) SR / MinSR normalisation: Python/tests/nqs/test_tdvp_matrix_free_regressions.py:18-151
    f = os.path.join(tests, "nqs", "test_tdvp_matrix_free_regressions.py")
    tr = _load(f)
    out["sr"] = {
        "source": "Python/tests/nqs/test_tdvp_matrix_free_regressions.py:18-151",
        "O": _cplx(_first_array_literal(_func(tr, "_wide_operator"))),
        "loss": _cplx(_first_array_literal(_func(tr, "_loss_vector"))),
        "shift_gram": _assign_literal(_func(tr, "test_matrix_free_standard_sr_uses_sample_normalization_for_wide_operator"), "shift"),
        "shift_minsr_solvers": _assign_literal(_func(tr, "test_jax_fisher_solvers_use_runtime_normalization_for_minsr_shape"), "shift"),
        "rtol": 2e-5,
    }

    # (2) estimator orientation + reweighting: test_nqs_generic_config_and_learning.py:337-499
    f = os.path.join(tests, "nqs", "test_nqs_generic_config_and_learning.py")
    tr = _load(f)
    fn = _func(tr, "test_complex_local_estimator_matches_dense_matrix_expectation")
    out["sigma_y_orientation"] = {
        "source": "Python/tests/nqs/test_nqs_generic_config_and_learning.py:337-371",
        "psi": _cplx(_assign_literal(fn, "psi")),
        "matrix": _cplx(_assign_literal(fn, "matrix")),
    }
    fn = _func(tr, "test_vmc_sample_prob_helper_matches_explicit_reweighting")
    out["reweighting"] = {
        "source": "Python/tests/nqs/test_nqs_generic_config_and_learning.py:425-443",
        "log_ansatz": _cplx(_assign_literal(fn, "log_ansatz")),
        "exponent": _assign_literal(fn, "log_prob_exponent"),
    }
    fn = _func(tr, "test_static_vmc_reweights_from_effective_sampling_beta")
    out["reweighting_beta"] = {
        "source": "Python/tests/nqs/test_nqs_generic_config_and_learning.py:459-499",
        "states": _assign_literal(fn, "states"),
        "mu": _assign_literal(fn, "mu"),
        "beta": _assign_literal(fn, "beta"),
        "logprob_fact": _assign_literal(fn, "logprob_fact"),
    }
    fn = _func(tr, "test_local_estimator_connected_state_chunking_preserves_result")
    out["chunking"] = {
        "source": "Python/tests/nqs/test_nqs_generic_config_and_learning.py:282-335",
        "params": _assign_literal(fn, "params"),
        "states": _assign_literal(fn, "states"),
    }

    # (3) RBM fast update inputs: Python/tests/nqs/test_rbm_fast_update.py:47-147
    f = os.path.join(tests, "nqs", "test_rbm_fast_update.py")
    tr = _load(f)
    fn = _func(tr, "test_rbm_log_psi_delta_cache_and_masked_updates_match_direct_eval")
    out["rbm_fast_update"] = {
        "source": "Python/tests/nqs/test_rbm_fast_update.py:111-147",
        "states": _assign_literal(fn, "states"),
        "indices": _assign_literal(fn, "indices"),
        "valid_mask": _assign_literal(fn, "valid_mask"),
        "n_hidden": 5,
        "rtol": 1e-6,
    }
    fn = _func(tr, "test_rbm_log_psi_delta_matches_direct_eval_single_flip")
    out["rbm_single_flip"] = {
        "source": "Python/tests/nqs/test_rbm_fast_update.py:47-61",
        "state": _assign_literal(fn, "state"),
        "flip": _assign_literal(fn, "update_info")[0],
    }

    # (4) integer operator encoding: Python/tests/algebra/test_custom_hamiltonian_workflows.py:75-87
    f = os.path.join(tests, "algebra", "test_custom_hamiltonian_workflows.py")
    tr = _load(f)
    fn = _func(tr, "test_operator_actions_on_integer_and_vector_states_are_stable")
    cases = {}
    for node in ast.walk(fn):
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Call):
            name = getattr(node.value.func, "id", "")
            if name in ("sigma_x_int_np", "sigma_z_int_np"):
                tgt = node.targets[0].elts[0].id.split("_")[0]
                cases[tgt] = {"op": name, "args": [ast.literal_eval(a) for a in node.value.args]}
        if isinstance(node, ast.Assert) and isinstance(node.test, ast.Compare):
            lhs = getattr(node.test.left, "id", "")
            for pref in ("sx", "sz"):
                if lhs == f"{pref}_states":
                    cases.setdefault(pref, {})["states"] = list(ast.literal_eval(node.test.comparators[0]))
                if lhs == f"{pref}_coeffs":
                    cases.setdefault(pref, {})["coeffs"] = list(ast.literal_eval(node.test.comparators[0]))
    out["int_operators"] = {
        "source": "Python/tests/algebra/test_custom_hamiltonian_workflows.py:75-87",
        "cases": cases,
    }

    # (5) two-site sigma^x normalisation: Python/tests/nqs/test_nqs_model_state_convention.py:136-147
    f = os.path.join(tests, "nqs", "test_nqs_model_state_convention.py")
    tr = _load(f)
    fn = _func(tr, "test_sigma_x_jax_respects_nonunit_binary_vector_convention")
    exp = None
    for node in ast.walk(fn):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", None) == "asarray":
            try:
                exp = ast.literal_eval(node.args[0])
            except ValueError:
                pass
    out["sigma_x_two_site"] = {
        "source": "Python/tests/nqs/test_nqs_model_state_convention.py:136-147",
        "coeff": exp[0] if isinstance(exp, list) and len(exp) == 1 else exp,
    }

    with open(args.out, "w", encoding="utf-8") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
