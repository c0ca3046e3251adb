"""Sweep-setting autotuner (cunibs_b200.tune): argument checks and the subject's defaults (no GPU)."""

from __future__ import annotations

import pytest

from cunibs_b200 import Subject
from cunibs_b200.synthetic import figure8_coil, sphere_head
from cunibs_b200.tune import autotune


@pytest.fixture(scope="module")
def subject():
    return Subject(sphere_head(12.0, 90.0, seed=0))


def test_sweep_defaults_are_validated(subject):
    assert subject.block_k_default == 8 and subject.overlap_blocks_per_sm == 2
    with pytest.raises(ValueError, match="block_k"):
        subject.set_sweep_defaults(block_k=17)
    with pytest.raises(ValueError, match="overlap"):
        subject.set_sweep_defaults(overlap_blocks_per_sm=0)
    subject.set_sweep_defaults(block_k=4)
    assert subject.block_k_default == 4
    subject.set_sweep_defaults(block_k=16)  # a block_k=None sweep may run wider than an explicit block_k
    assert subject.block_k_default == 16
    subject.set_sweep_defaults(block_k=8)


@pytest.mark.parametrize("kw, match", [(dict(widths=(0, 4)), "block widths"), (dict(widths=(32,)), "block widths"),
                                       (dict(overlaps=(17,)), "overlaps"), (dict(repeats=0), "repeats")])
def test_autotune_rejects_bad_candidates_before_any_work(subject, kw, match):
    with pytest.raises(ValueError, match=match):
        autotune(subject, figure8_coil(16), [], **kw)


def test_autotune_needs_placements(subject):
    with pytest.raises(ValueError, match="at least one placement"):
        autotune(subject, figure8_coil(16), [])


def test_simulate_subjects_rejects_a_shared_subject(subject):
    from cunibs_b200.batch import SubjectJob, simulate_subjects

    job = SubjectJob(subject, figure8_coil(16), [])
    with pytest.raises(ValueError, match="its own subject"):
        simulate_subjects([job, job])
