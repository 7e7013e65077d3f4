"""Autotuner for the packed persistent LM launch.

Picks, for a given packed batch, the number of warps per CTA (and the team size of
every robot class, which is 32 lanes: the kernel is built for one problem per warp)
by timing candidate launches of the real batch with CUDA events.  Results are cached
per batch signature (robot shapes, target counts, problem counts), so a serving loop
pays the search once.  Candidates: warps per CTA in {2, 4, 8}.
"""

from __future__ import annotations

import itertools

import torch

from .exceptions import KernelError

BR_ETOOBIG = -2  # include/br_b200.h: a launch shape above the library limit
_CACHE: dict = {}


def _team_choices(nv: int) -> list[int]:
    return [32]  # the kernel is built for 32-lane teams (see lm_solve.cu)


def signature(pk) -> tuple:
    return (tuple((m.njoints, m.nq, m.nv) for m in pk.models), tuple(pk.counts), pk.K, str(pk.device))


def tune(make_packed, settings, warps=(2, 4, 8), reps: int = 3, max_candidates: int = 24):
    """Return ``(team_sizes, warps_per_cta, ms)`` of the fastest candidate.

    ``make_packed(team_sizes, warps_per_cta)`` builds a ``PackedIK`` with its inputs set.
    """
    base = make_packed(None, 4)
    key = signature(base) + (int(getattr(settings, "precision", 0)),)
    if key in _CACHE:
        return _CACHE[key]
    choices = [_team_choices(m.nv) for m in base.models]
    cands = list(itertools.product(*choices))[:max_candidates]
    stream = torch.cuda.current_stream()
    best = None
    for teams in cands:
        for w in warps:
            try:
                pk = make_packed(list(teams), w)
                pk.solve(settings)  # warm-up
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    pk.solve(settings)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
            except KernelError as e:  # a shape the library refuses is skipped; any other error propagates
                if e.status != BR_ETOOBIG:
                    raise
                continue
            if best is None or ms < best[2]:
                best = (list(teams), w, ms)
    _CACHE[key] = best
    return best
