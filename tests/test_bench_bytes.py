"""The bench's algorithmic byte counts per kernel class (CPU).

Every class the step's event profiler reports (kStepKernelNames in csrc/gpu/state.cuh) must have a
nonzero count in both precisions, or its GB/s and roofline fraction would read as zero.  With the
two-ion sources, the mixed path has no cell-current pass in `prepare`: the face-candidate pass writes
the face terms of J (16 bytes per face) instead.
"""
import os
import re

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# entity counts in the ratios of a tetrahedral mesh (faces ~2 per cell, edges ~1.2, 4 faces per cell)
COUNTS = dict(nc=1000, nf=2000, ne=1170, c2f=4000, f2e=6000, e2f=6000, ec=6000, f2c=4000)


def step_classes():
    src = open(os.path.join(ROOT, "mpcns_uns_b200", "csrc", "gpu", "state.cuh")).read()
    body = re.search(r"kStepKernelNames\[KP_COUNT\]\s*=\s*\{([^}]*)\}", src).group(1)
    return re.findall(r'"(\w+)"', body)


def test_profiler_classes_are_the_ones_the_bench_counts():
    assert step_classes() == ["prepare", "cfl", "limited_gradients", "face_flux", "update", "face_candidate",
                              "edge_emf", "ct", "gyrate"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sources", [False, True])
def test_every_class_has_bytes(precision, sources):
    for k in step_classes():
        b = bench.algorithmic_bytes(k, COUNTS, 2, 2, precision, sources)
        if k == "gyrate" and not sources:
            assert b == 0          # no gyration without the two-ion sources
            continue
        per_cell = b / COUNTS["nc"]
        assert 20 < per_cell < 2000, (k, precision, sources, per_cell)


def test_mixed_sources_counts():
    c, nf = COUNTS, COUNTS["nf"]
    assert bench.algorithmic_bytes("prepare", c, 2, 2, "mixed", True) == bench.algorithmic_bytes("prepare", c, 2, 2, "mixed", False)
    assert (bench.algorithmic_bytes("face_candidate", c, 2, 2, "mixed", True)
            == bench.algorithmic_bytes("face_candidate", c, 2, 2, "mixed", False) + 16 * nf)
    # the FP64 path does run the cell-current pass inside its prepare class
    assert bench.algorithmic_bytes("prepare", c, 2, 2, "fp64", True) > bench.algorithmic_bytes("prepare", c, 2, 2, "fp64", False)
