"""Reinforcement-learning driver of the leader-follower task, the loop of the
reference's main_RL_leadFollow.cpp (app_main, lines 79-177) without the
smarties library: the caller's agent (any policy) supplies the actions.

Shape 0 is the leader (any body), shape 1 the agent, a StefanFish.  Every
action lasts half of the agent's current tail period
(getTimeToNextAct, main_RL_leadFollow.cpp:75-77); the state is
StefanFish::state relative to the leader (16 values), the reward the
agent's deformation-power efficiency EffPDefBnd, or -10 when the agent
leaves the region 0.5 < dX/L < 3, |dY/L| < 1 behind the leader
(isTerminal / getReward, :45-59); a non-finite state or reward ends the
episode with reward -1000 and a zero state (checkNaN, :61-73).
"""
import math

import numpy as np

from .abi import Cup2DError, ESTATE, Simulation

MAX_LEARN_STEPS = 200            # maxLearnStepPerSim (main_RL_leadFollow.cpp:89)
ACTION_LOW = (-1.0, -0.25)       # setActionScales bounds (:95-96)
ACTION_HIGH = (1.0, 0.25)


def is_terminal(agent, leader, length):
    """isTerminal (main_RL_leadFollow.cpp:45-50) on two shape-state dicts."""
    X = (agent["center_x"] - leader["center_x"]) / length
    Y = (agent["center_y"] - leader["center_y"]) / length
    return abs(Y) > 1 or X < 0.5 or X > 3


def reward_of(agent, leader, length):
    """getReward (main_RL_leadFollow.cpp:52-56)."""
    return -10.0 if is_terminal(agent, leader, length) else agent["EffPDefBnd"]


def check_nan(state, reward):
    """checkNaN (main_RL_leadFollow.cpp:61-73): (state, reward, trouble)."""
    if math.isnan(reward) or np.any(np.isnan(state)):
        return np.zeros_like(state), -1000.0, True
    return state, reward, False


class LeadFollow:
    """One simulation of the leader-follower task on the device pipeline.

    reset() -> state; step(action) -> (state, reward, done, info), with
    info["reason"] in {"running", "terminal", "nan", "last"}."""

    def __init__(self, argline, training=True, seed=0):
        self.sim = Simulation(argline)
        self.sim.init()
        if self.sim.ctx.nshapes < 2:
            raise Cup2DError(ESTATE, "the task needs a leader (shape 0) and an agent (shape 1)")
        self.training = training
        self.rng = np.random.default_rng(seed)
        self.length = [p.L for _, p in self.sim.shape_params][1]
        self.t = self.t_next = 0.0
        self.steps = 0

    # resetIC (main_RL_leadFollow.cpp:27-41)
    def _reset_ic(self):
        ctx, L = self.sim.ctx, self.length
        if self.training:
            SX = self.rng.uniform(0, 0.5)
            SY = self.rng.uniform(-0.25, 0.25)
            SA = self.rng.uniform(-20 / 180 * math.pi, 20 / 180 * math.pi)
        else:
            SX, SY, SA = 0.25, 0.0, 0.0
        p, a = ctx.shape(0), ctx.shape(1)
        C = (p["center_x"] + (1 + SX) * L, p["center_y"] + SY * L)
        p["com_y"] = p["center_y"] - (C[1] - p["center_y"])
        p["center_y"] = p["center_y"] - (C[1] - p["center_y"])
        a["com_x"], a["com_y"] = C
        a["orientation"] = SA
        ctx.set_shape(0, p)
        ctx.set_shape(1, a)

    def reset(self):
        """Simulation::reset, the randomised initial condition, the state."""
        self.sim.ctx.init()
        self._reset_ic()
        self.t = self.t_next = 0.0
        self.steps = 0
        return self.sim.ctx.fish_state(1, 0)

    def step(self, action):
        ctx = self.sim.ctx
        action = np.clip(np.asarray(action, dtype=np.float64), ACTION_LOW[:len(action)],
                         ACTION_HIGH[:len(action)])
        ctx.fish_act(1, self.t_next, action)
        self.t_next = self.t_next + ctx.fish_period(1) / 2
        over = False
        while self.t < self.t_next:
            dt = self.sim.calcMaxTimestep()
            self.t += dt
            if self.sim.advance(dt):
                raise Cup2DError(ESTATE, "the simulation reached -nsteps/-tend: leave both at 0")
            if is_terminal(ctx.shape(1), ctx.shape(0), self.length):
                over = True
                break
        self.steps += 1
        state = ctx.fish_state(1, 0)
        reward = reward_of(ctx.shape(1), ctx.shape(0), self.length)
        state, reward, bad = check_nan(state, reward)
        if over or bad:
            return state, reward, True, {"reason": "nan" if bad else "terminal"}
        if self.steps >= MAX_LEARN_STEPS:
            return state, reward, True, {"reason": "last"}
        return state, reward, False, {"reason": "running"}
