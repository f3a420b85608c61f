"""Host logic of the leader-follower driver (main_RL_leadFollow.cpp:45-77)
on plain values: the terminal region, the reward and the NaN guard."""
import numpy as np

from cubismup_2d_b200.rl import check_nan, is_terminal, reward_of


def _pose(x, y, eff=0.3):
    return {"center_x": x, "center_y": y, "EffPDefBnd": eff}


def test_terminal_region_and_reward():
    lead = _pose(0.3, 0.25)
    L = 0.1
    assert not is_terminal(_pose(0.3 + 1.0 * L, 0.25), lead, L)
    assert is_terminal(_pose(0.3 + 0.4 * L, 0.25), lead, L)         # X < 0.5
    assert is_terminal(_pose(0.3 + 3.1 * L, 0.25), lead, L)         # X > 3
    assert is_terminal(_pose(0.3 + 1.0 * L, 0.25 + 1.1 * L), lead, L)   # |Y| > 1
    assert reward_of(_pose(0.3 + 1.0 * L, 0.25, 0.42), lead, L) == 0.42
    assert reward_of(_pose(0.3 + 0.2 * L, 0.25, 0.42), lead, L) == -10.0


def test_nan_guard():
    s = np.arange(16, dtype=float)
    out, r, bad = check_nan(s, 0.5)
    assert not bad and r == 0.5 and np.array_equal(out, s)
    s[3] = np.nan
    out, r, bad = check_nan(s, 0.5)
    assert bad and r == -1000.0 and not np.any(out)
    out, r, bad = check_nan(np.zeros(16), float("nan"))
    assert bad and r == -1000.0
