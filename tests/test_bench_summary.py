"""The bench line's closing `summary` object (CPU): built from every leg the default run prints, without a
missing key, and short enough to survive a log cut to the line's last 1500 characters."""
import json

import bench


def _line():
    kern = {"s_per_solve": 0.5, "iterations": 300, "rel_res": 3.0e-4, "reorth_passes": 0}
    fd = {"switch_free": {"directions": 6, "max_rel_err": 9.4e-8},
          "crossing": {"directions": 16, "max_rel_err": 4.0e-5, "median_rel_err": 6.2e-6}}
    return {
        "ms_per_step": 10.99, "e2e": {"value": 9.3e8}, "roofline": {"frac": 0.67, "kernel": "update"},
        "clocks": {"sm_mhz": 1905.0}, "fp64": {"ms_per_step": 33.8, "speedup_mixed": 3.08, "clocks": {"sm_mhz": 1965.0}},
        "accuracy_mixed_vs_fp64": {"steps": 100, "U_all_rel_l2": 1.18e-7, "U0_rel_l2": 1.15e-7, "U1_rel_l2": 1.13e-4,
                                   "U0_perturbed_1e-7": 1.39e-7, "U1_perturbed_1e-7": 1.51e-4, "Phi_rel_l2": 3.96e-8,
                                   "div_b_max_rel_mixed": 8.05e-16, "div_b_max_rel_fp64": 9.84e-16},
        "gmres": {"fp64": dict(kern), "mixed": dict(kern, s_per_solve=0.39), "speedup_mixed": 1.3,
                  "ilu": {"max_it": 60, "ilu": {"s_per_solve": 0.73, "rel_res": 5.4e-4},
                          "jacobi": {"s_per_solve": 0.11, "rel_res": 8.4e-4}, "factor_ms": 62.3, "apply_ms": 9.1}},
        "semi_implicit": {"ms_per_step": 38.4, "iterations": [5, 5, 5], "rel_res": [4.1e-9, 3.9e-9, 4.0e-9]},
        "config1": {"fp64": {"ms_per_step": 0.35}, "mixed": {"error": "reported, not raised"}},
        "adjoint": {"forward_s": 0.2, "forward_plus_backward_over_forward": 3.79, "dot_test_rel_err_max": 2.7e-15,
                    "fd": {"h=1e-06": fd, "h=1e-07": fd}},
        "ten_ion": {"mixed": {"ms_per_step": 105.5}, "fp64": {"ms_per_step": 325.5},
                    "accuracy_mixed_vs_fp64": {"U_all_rel_l2": 1.9e-9}},
    }


def test_summary_of_every_leg():
    sm = bench.summary(_line())
    for key in ("acc", "gmres", "semi_implicit", "adjoint", "ten_ion", "config1"):
        assert key in sm, key
    assert sm["config1"] == {"fp64": 0.35, "mixed": None}
    assert sm["gmres"]["ilu"]["factor_apply_ms"] == [62.3, 9.1]
    assert sm["semi_implicit"] == {"ms": 38.4, "it": [5, 5, 5], "rel_res": 4.1e-9}
    assert len(json.dumps({"summary": sm})) < 1400


def test_summary_without_the_optional_legs():
    out = _line()
    for key in ("accuracy_mixed_vs_fp64", "gmres", "semi_implicit", "adjoint", "ten_ion", "config1"):
        out.pop(key)
    sm = bench.summary(out)
    assert set(sm) == {"mixed_ms", "fp64_ms", "speedup_mixed", "e2e", "roofline_frac", "roofline_kernel", "clocks_mhz"}
