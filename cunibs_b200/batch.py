"""Several subjects' sweeps at once on one GPU.

Every subject owns a native context with its own streams (a solve stream and a preparation
stream), so the sweeps of subjects of uneven mesh size can run side by side: one host thread per
subject drives its pipelined ``Subject.iter_simulate`` (the native calls release the interpreter
lock), and the GPU interleaves their latency-bound solves and FMA-bound dA/dt kernels. Each
subject's results are bitwise those of its sweep alone: nothing is shared between contexts.
"""

from __future__ import annotations

import threading
from collections.abc import Sequence
from dataclasses import dataclass, field


@dataclass
class SubjectJob:
    """One subject's sweep: ``Subject.iter_simulate(coil, placements, didt, **options)``."""

    subject: object
    coil: object
    placements: Sequence
    didt: float = 1e6
    options: dict = field(default_factory=dict)


def simulate_subjects(jobs: Sequence[SubjectJob]) -> list[list]:
    """Run the jobs concurrently, one host thread each, and return every job's FieldResults in
    order. The subjects must be distinct (one subject's calls are serialised by its own lock). The
    first error of any job is raised after all threads have finished."""
    jobs = list(jobs)
    if len({id(j.subject) for j in jobs}) != len(jobs):
        raise ValueError("each job needs its own subject")
    for j in jobs:
        j.subject.context  # build the contexts before the threads start  # noqa: B018
    results: list[list | None] = [None] * len(jobs)
    errors: list[BaseException | None] = [None] * len(jobs)

    def run(i: int) -> None:
        j = jobs[i]
        try:
            results[i] = list(j.subject.iter_simulate(j.coil, j.placements, j.didt, **j.options))
        except BaseException as exc:  # noqa: BLE001 - re-raised in the caller's thread
            errors[i] = exc

    threads = [threading.Thread(target=run, args=(i,), name=f"cunibs-subject-{i}") for i in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for exc in errors:
        if exc is not None:
            raise exc
    return results  # type: ignore[return-value]
