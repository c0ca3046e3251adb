"""Several subjects swept at once (cunibs_b200.batch). Needs a B200.

Subjects of uneven size run side by side from one host thread each; each subject's results must be
bitwise those of its sweep alone.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject
from cunibs_b200.batch import SubjectJob, simulate_subjects
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu


def _sites(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        th, ph = rng.uniform(0.0, 0.5), rng.uniform(0.0, 2 * np.pi)
        c = 90.0 * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        out.append(Placement(c, c + [-50.0 * np.sin(ph), 50.0 * np.cos(ph), 0.0]))
    return out


def test_concurrent_subjects_match_their_sweeps_alone():
    coil = figure8_coil(64)
    subjects = [Subject(sphere_head(h, 90.0, jitter_mm=0.3, seed=s), tolerance=1e-8)
                for h, s in ((6.0, 1), (8.0, 2), (5.0, 3))]
    jobs = [SubjectJob(subj, coil, _sites(10, i), options=dict(magnitude=True)) for i, subj in enumerate(subjects)]
    alone = [[r.magnE for r in j.subject.iter_simulate(j.coil, j.placements, magnitude=True)] for j in jobs]
    together = simulate_subjects(jobs)
    for a, t in zip(alone, together):
        assert len(t) == len(a)
        for x, r in zip(a, t):
            np.testing.assert_array_equal(r.magnE, x)
    with pytest.raises(ValueError, match="its own subject"):
        simulate_subjects([jobs[0], jobs[0]])
    for s in subjects:
        s.free()
