"""BatchAtariGpuEnv: the reference's batched RL caller on the B200 core.

Mirrors src/rl4burn_env.rs:269-380: N parallel instances of one ROM, a single
discrete action broadcast to all of them, frameskip (action repeat, default 4)
through step_multi, truncation after max_steps (default 108,000), reward 0 and
terminated false (the reference extracts no reward).  Observations are the
N x 128 RAM bytes as f32 / 255, flattened to N*128 — produced on the device
into a torch CUDA tensor (fa_obs_to_unit_f32) instead of on the host.

with_reward(spec) adds what the reference lacks: per-instance rewards (score
change) and episode flags (terminal test, life lost) decoded from RAM on the
device (fa_obs_reward), returned as CUDA tensors of shape (N,).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import BatchAtariGpu, RewardSpec, _check, _vp, lib, obs_reward

NUM_ACTIONS = 18            # src/rl4burn_env.rs:26
DEFAULT_MAX_STEPS = 108_000  # :29
DEFAULT_FRAMESKIP = 4        # :32


@dataclass
class Step:
    observation: "object"    # torch.Tensor, float32, shape (N*128,), on the device
    reward: "object"         # 0.0, or with a reward spec a float32 tensor (N,)
    terminated: "object"     # False, or with a reward spec a bool tensor (N,) (terminal test)
    truncated: bool
    life_lost: "object" = None   # with a reward spec: bool tensor (N,)


class BatchAtariGpuEnv:
    def __init__(self, rom: bytes, n: int, device: int = 0):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        self.gpu = BatchAtariGpu(rom, n)
        self.rom = bytes(rom)
        self.n = int(n)
        self.step_count = 0
        self.max_steps = DEFAULT_MAX_STEPS
        self.frameskip = DEFAULT_FRAMESKIP
        self._actions = torch.zeros(self.n * 64, dtype=torch.uint8, device=self.device)
        self._obs_u8 = torch.zeros(self.n * 128, dtype=torch.uint8, device=self.device)
        self._obs = torch.zeros(self.n * 128, dtype=torch.float32, device=self.device)
        self.reward_spec = None

    def with_reward(self, spec: RewardSpec) -> "BatchAtariGpuEnv":
        """Score, lives and end-of-episode positions in RAM (fa_obs_reward)."""
        t = self.torch
        self.reward_spec = spec
        self._score = t.zeros(self.n, dtype=t.int32, device=self.device)
        self._lives = t.zeros(self.n, dtype=t.int32, device=self.device)
        self._reward = t.zeros(self.n, dtype=t.float32, device=self.device)
        self._flags = t.zeros(self.n, dtype=t.uint8, device=self.device)
        return self

    def with_reward_table(self, table, game: str = None) -> "BatchAtariGpuEnv":
        """The reward spec of this env's game from a reward table (a path or a
        rewards.RewardTable): by `game` name, else by the ROM's SHA-256."""
        from .rewards import RewardTable
        tab = table if isinstance(table, RewardTable) else RewardTable.load(table)
        spec = tab.for_game(game) if game is not None else tab.for_rom(self.rom)
        if spec is None:
            raise KeyError("no entry of the reward table matches this ROM; name the game")
        return self.with_reward(spec)

    def _rewards(self, init: bool):
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        obs_reward(self._obs_u8.data_ptr(), self.n, self.reward_spec, init, self._score.data_ptr(),
                   self._lives.data_ptr(), self._reward.data_ptr(), self._flags.data_ptr(), stream)

    # builder methods (src/rl4burn_env.rs:298-313)
    def with_max_steps(self, max_steps: int) -> "BatchAtariGpuEnv":
        self.max_steps = int(max_steps)
        return self

    def with_frameskip(self, frameskip: int) -> "BatchAtariGpuEnv":
        if frameskip < 1:
            raise ValueError("frameskip must be >= 1")
        self.frameskip = int(frameskip)
        if self.frameskip * self.n > self._actions.numel():
            self._actions = self.torch.zeros(self.frameskip * self.n, dtype=self.torch.uint8, device=self.device)
        return self

    def with_sorted(self, sorted_: bool) -> "BatchAtariGpuEnv":
        self.gpu.set_sorted(sorted_)
        return self

    def num_envs(self) -> int:
        return self.n

    def observation_space(self):
        return ("Box", 0.0, 1.0, self.n * 128)

    def action_space(self):
        return ("Discrete", NUM_ACTIONS)

    def _normalise(self):
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        _check(lib().fa_obs_to_unit_f32(_vp(self._obs_u8.data_ptr()), _vp(self._obs.data_ptr()),
                                         self._obs.numel(), _vp(stream or None)))
        return self._obs

    def reset(self):
        """src/rl4burn_env.rs:331-338: step counter 0, RAM after reset."""
        self.step_count = 0
        ram = self.gpu.reset()
        self._obs_u8.copy_(self.torch.from_numpy(np.ascontiguousarray(ram).reshape(-1)))
        if self.reward_spec is not None:
            self._rewards(init=True)
        return self._normalise().clone()

    def step(self, action: int) -> Step:
        """src/rl4burn_env.rs:340-367: broadcast, frameskip, truncation."""
        k = self.frameskip
        acts = self._actions[: k * self.n]
        acts.fill_(int(action) & 0xFF)
        self.torch.cuda.current_stream(self.device).synchronize()
        self.gpu.step_multi_async(acts.data_ptr(), k, self._obs_u8.data_ptr())
        self.gpu.synchronize()
        obs = self._normalise().clone()
        self.step_count += 1
        truncated = self.max_steps > 0 and self.step_count >= self.max_steps
        if self.reward_spec is None:
            return Step(obs, 0.0, False, truncated)
        self._rewards(init=False)
        f = self._flags
        return Step(obs, self._reward.clone(), (f & 1).bool(), truncated, (f & 2).bool())

    def close(self):
        self.gpu.close()
