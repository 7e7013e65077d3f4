"""The LM's level schedule over the DOF tree (``br_dof_schedule``, host code of the library).

Interprets the schedule in float64 numpy exactly as ``lm_solve_kernel``'s level path reads
it (tasks of a level, pivots, back substitution by depth) and checks the solution of
``(A + damp I) x = -g`` against a dense solve for random matrices with the DOF tree's
sparsity (``A[i, j] != 0`` only when one of i, j is an ancestor of the other), plus the
properties the kernel relies on: within a level every destination is written by one
task, and no row a task reads is written in the same level."""

import numpy as np
import pytest

from betterrobot_b200 import synthetic as syn
from betterrobot_b200.tree import TreeArrays

pytestmark = pytest.mark.filterwarnings("ignore")


def _lib():
    from betterrobot_b200 import _lib
    try:
        return _lib.load()
    except Exception as e:  # library not built here
        pytest.skip(str(e))


def _tree(dof_parent):
    nv = len(dof_parent)
    dep, anc, rowoff, nl = [0] * nv, [[] for _ in range(nv)], [0] * (nv + 1), 0
    for c, p in enumerate(dof_parent):
        dep[c] = 0 if p < 0 else dep[p] + 1
        anc[c] = [] if p < 0 else anc[p] + [p]
        rowoff[c] = nl
        nl += dep[c] + 1
    rowoff[nv] = nl
    return dep, anc, rowoff


def _schedule(dof_parent):
    lib = _lib()
    dp = np.ascontiguousarray(dof_parent, dtype=np.int32)
    n = lib.br_dof_schedule(dp.ctypes.data, len(dp), None, 0)
    assert n > 0
    out = np.zeros(n, np.uint32)
    assert lib.br_dof_schedule(dp.ctypes.data, len(dp), out.ctypes.data, n) == n
    return out


def _decode(s):
    nlev, ntask, nextra, ndl = (int(v) for v in s[:4])
    starts = s[4:5 + nlev].astype(np.int64)
    toff = (5 + nlev + 3) & ~3
    tasks = s[toff:toff + 4 * ntask].reshape(ntask, 4).astype(np.int64)
    extra = s[toff + 4 * ntask:toff + 4 * ntask + 2 * nextra].reshape(nextra, 2).astype(np.int64)
    return nlev, ndl, starts, tasks, extra


def _contribs(tk, extra):
    out = [(tk[1] & 0xffff, tk[1] >> 16, tk[2] & 0xffff)]
    first, n = tk[2] >> 16, tk[0] >> 16
    out += [(e[0] & 0xffff, e[0] >> 16, e[1]) for e in extra[first:first + n]]
    return out


def _solve(s, dof_parent, A, g, damp):
    nv = len(dof_parent)
    dep, anc, rowoff = _tree(dof_parent)
    nL = rowoff[nv]
    m = np.zeros(nL + nv)
    for c in range(nv):
        for a, p in enumerate(anc[c]):
            m[rowoff[c] + a] = A[c, p]
        m[rowoff[c] + dep[c]] = A[c, c]
    m[nL:] = -g
    nlev, ndl, starts, tasks, extra = _decode(s)
    # leaves' pivots are final from the start; a non-leaf's is stored by the flagged task
    dinv = np.array([1.0 / (m[rowoff[i] + dep[i]] + damp) for i in range(nv)])
    for lev in range(nlev):
        for tk in tasks[starts[lev]:starts[lev + 1]]:
            acc = m[tk[0] & 0xffff]
            for a, b, k in _contribs(tk, extra):
                acc -= m[a] * dinv[k] * m[b]
            m[tk[0] & 0xffff] = acc
            if tk[3]:
                dinv[tk[3] - 1] = 1.0 / (acc + damp)
    piv = np.array([m[rowoff[i] + dep[i]] + damp for i in range(nv)])
    assert np.allclose(dinv, 1.0 / piv, rtol=0, atol=0)
    assert (piv > 0).all()
    x = np.zeros(nv)
    for dl in range(ndl):
        for i in range(nv):
            if dep[i] == dl:
                acc = m[nL + i] - sum(m[rowoff[i] + a] * x[anc[i][a]] for a in range(dl))
                x[i] = acc / piv[i]
    return x


def _random_tree_matrix(dof_parent, rng, n_terms=12):
    nv = len(dof_parent)
    _, anc, _ = _tree(dof_parent)
    A = np.zeros((nv, nv))
    for _ in range(n_terms):
        c = int(rng.integers(nv))
        sup = anc[c] + [c]
        for _ in range(6):
            v = np.zeros(nv)
            v[sup] = rng.normal(size=len(sup))
            A += np.outer(v, v)
    return A


def _dof_parents():
    specs = {"chain7": syn.chain_spec(), "humanoid": syn.humanoid_spec(), "dual_arm": syn.dual_arm_spec()}
    if hasattr(syn, "mixed_spec"):
        specs["mixed"] = syn.mixed_spec()
    out = {n: TreeArrays(syn.model_from_spec(sp)).dof_parent for n, sp in specs.items()}
    out["forest"] = np.array([-1, 0, 1, -1, 3, -1], np.int32)
    out["star"] = np.array([-1, 0, 0, 0, 0, 0, 0, 1, 2, 3], np.int32)
    return out


@pytest.mark.parametrize("name", ["chain7", "humanoid", "dual_arm", "mixed", "forest", "star"])
def test_schedule_solves_tree_system(name):
    parents = _dof_parents()
    if name not in parents:
        pytest.skip("no such synthetic robot")
    dp = parents[name]
    s = _schedule(dp)
    rng = np.random.default_rng(len(dp))
    for damp in (1e-3, 1.0):
        A = _random_tree_matrix(dp, rng)
        g = rng.normal(size=len(dp))
        x = _solve(s, dp, A, g, damp)
        ref = np.linalg.solve(A + damp * np.eye(len(dp)), -g)
        assert np.abs(x - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("name", ["humanoid", "dual_arm", "star"])
def test_schedule_levels_are_race_free(name):
    dp = _dof_parents()[name]
    nv = len(dp)
    dep, anc, rowoff = _tree(dp)
    nL = rowoff[nv]
    row_of = np.zeros(nL + nv, np.int64)
    for c in range(nv):
        row_of[rowoff[c]:rowoff[c + 1]] = c
        row_of[nL + c] = c
    nlev, ndl, starts, tasks, extra = _decode(_schedule(dp))
    assert ndl == max(dep) + 1
    parents = set(int(p) for p in dp if p >= 0)
    final_later = set(parents)        # non-leaf DOFs whose pivot is not final yet
    assert int((tasks[:, 3] != 0).sum()) == len(parents)
    seen = 0
    for lev in range(nlev):
        lt = tasks[starts[lev]:starts[lev + 1]]
        dsts = [int(t[0] & 0xffff) for t in lt]
        assert len(dsts) == len(set(dsts))
        written = {int(row_of[d]) for d in dsts}
        read = {int(row_of[x]) for t in lt for a, b, k in _contribs(t, extra) for x in (a, b)}
        read |= {int(k) for t in lt for a, b, k in _contribs(t, extra)}   # pivots read
        assert not (written & read)
        # a pivot is read only after the level that finalised it
        for t in lt:
            for a, b, k in _contribs(t, extra):
                assert k not in final_later, (k, lev)
        for t in lt:
            if t[3]:
                c = int(t[3]) - 1
                assert int(t[0] & 0xffff) == rowoff[c] + dep[c]
                final_later.discard(c)
        seen += sum(1 + int(t[0] >> 16) for t in lt)
    # one contribution per (DOF, ancestor pair) plus one per (DOF, ancestor) for the right-hand side
    assert seen == sum(d * (d + 1) // 2 + d for d in dep)


def _trunk(dof_parent, kmax=6):
    """The float64 LM variants' register trunk (``lm_solve.cu``): the largest n <= 6 with DOFs
    0..n-1 a chain from the root and every other DOF below DOF n - 1; 0 when n < 2."""
    dp = [int(p) for p in dof_parent]
    nv = len(dp)
    _, anc, _ = _tree(dp)
    for n in range(min(nv, kmax), 1, -1):
        if dp[0] < 0 and all(dp[c] == c - 1 for c in range(1, n)) and all(n - 1 in anc[c] for c in range(n, nv)):
            return n
    return 0


@pytest.mark.parametrize("name", ["chain7", "humanoid", "dual_arm", "mixed", "forest", "star"])
def test_schedule_ends_with_the_trunk(name):
    """The kernel skips the schedule's last n levels for a trunk of n DOFs and eliminates
    n - 1, ..., 0 itself in registers, entry (i, j) <- fma(-(L_ki / d_k), L_kj, .): those
    levels must hold exactly that, one DOF per level, one contribution per entry."""
    parents = _dof_parents()
    if name not in parents:
        pytest.skip("no such robot in the synthetic module")
    dp = parents[name]
    n = _trunk(dp)
    expect = {"chain7": 6, "humanoid": 6, "dual_arm": 0, "forest": 0, "star": 0}
    if name in expect:
        assert n == expect[name]
    if n == 0:
        return
    nlev, _, starts, tasks, extra = _decode(_schedule(dp))
    _, _, rowoff = _tree(dp)
    zoff = rowoff[len(dp)]
    tri = lambda i: i * (i + 1) // 2  # noqa: E731
    for step, lev in enumerate(range(nlev - n, nlev)):
        k = n - 1 - step
        seen = set()
        for tk in tasks[starts[lev]:starts[lev + 1]]:
            cs = _contribs(tk, extra)
            assert len(cs) == 1
            a, b, d = cs[0]
            dst = int(tk[0] & 0xffff)
            assert d == k and dst not in seen
            seen.add(dst)
            if dst < zoff:                       # entry (i, j) of a trunk row, i < k
                i = max(r for r in range(k) if tri(r) <= dst)
                j = dst - tri(i)
                assert (a, b) == (tri(k) + i, tri(k) + j)
            else:                                # right-hand side of trunk DOF i < k
                i = dst - zoff
                assert i < k and (a, b) == (tri(k) + i, zoff + k)
        assert len(seen) == tri(k) + k           # every entry of rows 0..k-1 and their z


def test_schedule_rejects_bad_parents():
    lib = _lib()
    bad = np.array([-1, 1], np.int32)   # a DOF whose parent is not earlier
    assert lib.br_dof_schedule(bad.ctypes.data, 2, None, 0) < 0
    big = np.zeros(65, np.int32)
    assert lib.br_dof_schedule(big.ctypes.data, 65, None, 0) < 0


def test_schedule_at_the_size_limit():
    """A 62-DOF serial chain (64 joints with the universe and root) and a 64-DOF binary-ish tree."""
    chain = np.arange(-1, 61, dtype=np.int32)                 # c's parent is c - 1
    tree = np.array([-1] + [(c - 1) // 2 for c in range(1, 64)], np.int32)
    rng = np.random.default_rng(5)
    for dp in (chain, tree):
        s = _schedule(dp)
        A = _random_tree_matrix(dp, rng, n_terms=20)
        g = rng.normal(size=len(dp))
        x = _solve(s, dp, A, g, 1e-2)
        ref = np.linalg.solve(A + 1e-2 * np.eye(len(dp)), -g)
        assert np.abs(x - ref).max() <= 1e-8 * max(1.0, np.abs(ref).max())
