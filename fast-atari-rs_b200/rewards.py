"""Per-game reward tables: where each game keeps its score, lives and end
flag in RAM, loaded from a file into RewardSpec records for fa_obs_reward.

The reference returns reward 0 and never terminates (src/atari.rs:348,
src/rl4burn_env.rs:123); the addresses are per-game knowledge that no ROM
carries, so the caller supplies them in a table like this one (JSON):

    {
      "format": "fast-atari reward table 1",
      "games": {
        "<game name>": {
          "rom_sha256": "<hex digest of the ROM bytes>",      (optional)
          "score": ["0xD5", "0xD6"],                          RAM addresses, most significant byte first (1-4)
          "bcd": true,                                        score bytes are BCD (default true)
          "lives": {"addr": "0xBA", "mask": "0x0F", "shift": 0},       (optional)
          "terminal": {"addr": "0x80", "mask": "0x80", "value": "0x80"} (optional)
        }
      }
    }

Addresses are the game's RAM addresses $80-$FF (or offsets 0-127 into the
observation); numbers may be JSON integers or "0x.." strings.  The reward of
a step is the decoded score minus the previous step's; lives decode as
(RAM[addr] & mask) >> shift, and a drop raises FA_EPISODE_LIFE_LOST; the
episode ends (FA_EPISODE_TERMINAL) when RAM[addr] & mask == value.  A game
with no score entry yields reward 0, as the reference does.
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path
from typing import Dict, Optional, Union

from . import RewardSpec

FORMAT = "fast-atari reward table 1"


def _num(v, what: str) -> int:
    if isinstance(v, bool) or not isinstance(v, (int, str)):
        raise ValueError(f"{what}: expected an integer or a '0x..' string, got {v!r}")
    x = int(v, 0) if isinstance(v, str) else v
    if not 0 <= x <= 0xFF:
        raise ValueError(f"{what}: {x:#x} is not a byte")
    return x


def _ram(v, what: str) -> int:
    """A RAM address $80-$FF or an observation offset 0-127, as an offset."""
    x = _num(v, what)
    return x - 0x80 if x >= 0x80 else x


def spec_from_entry(entry: dict, name: str = "game") -> RewardSpec:
    """One game's table entry as a RewardSpec (validated)."""
    unknown = set(entry) - {"rom_sha256", "score", "bcd", "lives", "terminal", "comment"}
    if unknown:
        raise ValueError(f"{name}: unknown keys {sorted(unknown)}")
    score = [_ram(a, f"{name}.score[{i}]") for i, a in enumerate(entry.get("score", []))]
    if len(score) > 4:
        raise ValueError(f"{name}: at most 4 score bytes")
    lives = terminal = None
    if "lives" in entry:
        lv = entry["lives"]
        shift = int(lv.get("shift", 0))
        if not 0 <= shift <= 7:
            raise ValueError(f"{name}.lives.shift must be 0-7")
        lives = (_ram(lv["addr"], f"{name}.lives.addr"), _num(lv.get("mask", 0xFF), f"{name}.lives.mask"), shift)
    if "terminal" in entry:
        tm = entry["terminal"]
        terminal = (_ram(tm["addr"], f"{name}.terminal.addr"), _num(tm.get("mask", 0xFF), f"{name}.terminal.mask"),
                    _num(tm["value"], f"{name}.terminal.value"))
    return RewardSpec.make(score=score, bcd=bool(entry.get("bcd", True)), lives=lives, terminal=terminal)


class RewardTable:
    """A loaded reward table: specs by game name, and by ROM digest where the
    entry gives one."""

    def __init__(self, data: dict):
        if data.get("format") != FORMAT:
            raise ValueError(f"not a reward table (format must be {FORMAT!r})")
        games = data.get("games")
        if not isinstance(games, dict):
            raise ValueError("a reward table needs a 'games' object")
        self.specs: Dict[str, RewardSpec] = {}
        self.by_sha256: Dict[str, str] = {}
        for name, entry in games.items():
            self.specs[name] = spec_from_entry(entry, name)
            if "rom_sha256" in entry:
                self.by_sha256[str(entry["rom_sha256"]).lower()] = name

    @classmethod
    def load(cls, path: Union[str, Path]) -> "RewardTable":
        return cls(json.loads(Path(path).read_text()))

    def for_game(self, name: str) -> RewardSpec:
        return self.specs[name]

    def for_rom(self, rom: bytes) -> Optional[RewardSpec]:
        """The spec whose rom_sha256 matches these ROM bytes, or None."""
        name = self.by_sha256.get(hashlib.sha256(bytes(rom)).hexdigest())
        return self.specs[name] if name else None
