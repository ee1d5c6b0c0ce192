"""The oracle's fixpoint check (used on full-size device results) against
the oracle's own solve, and its detection of a planted mistake."""
from __future__ import annotations

import numpy as np

from oracle import ora


def test_fixpoint_check_accepts_solution_and_catches_a_planted_mistake():
    from gpuequiv_b200 import synth
    row, col, wt, att = synth.scaled_stress_game(5, 20_000, 100_000)
    sol = ora.run_game(6, 3, row, col, wt, att, ora.standard_reach(row, att))
    assert ora.check_fixpoint(row, col, wt, att, sol.offsets, sol.data) == (0, None)
    o = sol.offsets.astype(np.int64)
    d = sol.data
    # drop one energy of the first position holding two or more
    v = int(np.nonzero(np.diff(o) >= 2)[0][0])
    keep = np.ones(len(d), bool)
    keep[o[v]] = False
    o2 = o.copy()
    o2[v + 1:] -= 1
    assert ora.check_fixpoint(row, col, wt, att, o2.astype(np.uint64), d[keep]) == (1, v)
    # the initial state ({0} at the standard reach, empty elsewhere) is not a
    # fixpoint: the reach's predecessors change in the first step
    reach = ora.standard_reach(row, att)
    cnt = np.zeros(len(o) - 1, np.uint64)
    cnt[reach] = 1
    o0 = np.zeros(len(o), np.uint64)
    np.cumsum(cnt, out=o0[1:])
    n_bad, first = ora.check_fixpoint(row, col, wt, att, o0, np.zeros(len(reach), np.uint32))
    assert n_bad > 0 and first is not None
