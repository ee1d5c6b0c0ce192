"""The schedule-independent byte floor B_min = 4(n+1) + 8m + n +
sum_v 4|A*_v|(1 + indeg v) that the bench reports beside the roofline: the
library's host formula (gpuequiv_b200.b_min) against the oracle's
(ora_b_min) on the final lists of oracle solves, and on a game worked by
hand."""
import numpy as np

from oracle import ora


def test_hand_worked_game():
    import gpuequiv_b200 as geq
    # 0 (attacker) -> 1, 2 (defender sinks): lists {0}, {0}; 0 gets {e}
    g = geq.GameGraph(3, [(0, 1, [-1]), (0, 2, [0, -1])], [True, False, False], geq.EnergyConf.STANDARD)
    offs = np.array([0, 2, 3, 4], np.uint64)  # |A0| = 2, |A1| = |A2| = 1
    # 4*4 + 8*2 + 3 + 4*(2*(1+0) + 1*(1+1) + 1*(1+1)) = 16 + 16 + 3 + 24
    assert geq.b_min(g, offs) == 59
    assert ora.b_min(g.row_offsets, g.column_indices, offs) == 59


def test_random_games_match_the_oracle():
    import gpuequiv_b200 as geq
    rng = np.random.default_rng(11)
    for _ in range(20):
        n = int(rng.integers(2, 60))
        m = int(rng.integers(0, 3 * n))
        src = np.sort(rng.integers(0, n, m))
        dst = rng.integers(0, n, m)
        row = np.zeros(n + 1, np.uint32)
        np.add.at(row, src + 1, 1)
        row = np.cumsum(row).astype(np.uint32)
        wt = np.zeros(m, np.uint32)  # zero updates
        att = (rng.random(n) < 0.5).astype(np.uint8)
        g = geq.GameGraph.from_csr(row, dst.astype(np.uint32), wt, att, geq.EnergyConf.STANDARD)
        sol = ora.run_game(6, 3, row, dst.astype(np.uint32), wt, att, ora.standard_reach(row, att))
        assert geq.b_min(g, sol.offsets) == ora.b_min(row, dst, sol.offsets)
