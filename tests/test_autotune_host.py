"""The LM autotuner's host logic on the CPU (``betterrobot_b200.autotune``), with the CUDA
event clock replaced by a counter that each fake launch advances by its cost: the fastest
candidate wins, shapes the library refuses (``BR_ETOOBIG``) are skipped, any other kernel
error propagates, and a second call with the same batch signature is served from the cache.
"""

from types import SimpleNamespace

import pytest
import torch

from betterrobot_b200 import autotune
from betterrobot_b200.exceptions import KernelError


class _Clock:
    now = 0.0


class _Event:
    def __init__(self, enable_timing=True):
        self.at = None

    def record(self, stream=None):
        self.at = _Clock.now

    def elapsed_time(self, end):
        return end.at - self.at


class _Packed:
    """Stands in for ``PackedIK``: its shape fields, and a solve that costs ``cost`` ms."""

    def __init__(self, models, counts, warps, cost):
        self.models, self.counts, self.K, self.device = models, counts, 6, "cuda:0"
        self.warps, self.cost = warps, cost

    def solve(self, settings):
        c = self.cost[self.warps]
        if isinstance(c, Exception):
            raise c
        _Clock.now += c


@pytest.fixture
def fake_cuda(monkeypatch):
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "current_stream", lambda *a, **k: None)
    monkeypatch.setattr(autotune, "_CACHE", {})


def _maker(cost, counts, calls):
    models = [SimpleNamespace(njoints=32, nq=37, nv=36), SimpleNamespace(njoints=8, nq=7, nv=7)]

    def make(teams, warps):
        calls.append((None if teams is None else tuple(teams), warps))
        return _Packed(models, counts, warps, cost)
    return make


def test_fastest_candidate_refused_shapes_skipped_and_cached(fake_cuda):
    calls = []
    cost = {2: 1.0, 4: 0.5, 8: KernelError("shared memory", autotune.BR_ETOOBIG)}
    settings = SimpleNamespace(precision=0)
    teams, warps, ms = autotune.tune(_maker(cost, [10, 20], calls), settings)
    assert teams == [32, 32] and warps == 4 and ms == pytest.approx(0.5)
    n = len(calls)
    assert autotune.tune(_maker(cost, [10, 20], calls), settings) == (teams, warps, ms)
    assert len(calls) == n + 1                # only the signature probe: the result is cached
    # another batch signature (problem counts) or precision is tuned again
    cost2 = {2: 0.25, 4: 0.5, 8: 0.75}
    assert autotune.tune(_maker(cost2, [10, 21], calls), settings)[1] == 2
    assert autotune.tune(_maker(cost2, [10, 20], calls), SimpleNamespace(precision=1))[1] == 2


def test_other_kernel_errors_propagate(fake_cuda):
    cost = {2: 1.0, 4: KernelError("invalid argument", -1), 8: 0.5}
    with pytest.raises(KernelError):
        autotune.tune(_maker(cost, [4, 4], []), SimpleNamespace(precision=0))
