"""Reward tables (fast_atari_b200.rewards): the JSON format, its checks, and
lookup by game name or ROM digest.  CPU only; the GPU extraction itself is
tested in test_gpu_env.py."""
import hashlib
import json

import pytest

from fa_pkg import ROOT, carts, fa
from fast_atari_b200 import rewards

TABLE = ROOT / "fast-atari-rs_b200" / "reward_tables" / "synthetic_carts.json"


def test_shipped_table_loads_and_matches_roms():
    tab = rewards.RewardTable.load(TABLE)
    sp = tab.for_rom(carts.divergence_cart().rom)
    assert sp is not None and sp is tab.for_game("divergence_8k_f8")
    assert list(sp.score_addr[:3]) == [3, 4, 5] and sp.score_bytes == 3 and sp.score_bcd == 1
    assert (sp.lives_addr, sp.lives_mask, sp.lives_shift) == (7, 0x0C, 2)
    assert (sp.terminal_addr, sp.terminal_mask, sp.terminal_value) == (9, 0x80, 0x80)
    sp2 = tab.for_rom(carts.mixed_carts()[2].rom)
    assert sp2.score_bytes == 4 and sp2.score_bcd == 0 and sp2.lives_mask == 0 and sp2.terminal_mask == 0
    assert tab.for_rom(carts.plain_cart().rom) is None


def _table(entry):
    return {"format": rewards.FORMAT, "games": {"g": entry}}


@pytest.mark.parametrize("entry,msg", [
    ({"score": ["0x80"] * 5}, "at most 4"),
    ({"score": ["0x100"]}, "not a byte"),
    ({"score": [True]}, "integer"),
    ({"scores": ["0x80"]}, "unknown keys"),
    ({"lives": {"addr": "0x90", "shift": 9}}, "shift"),
])
def test_bad_entries_are_refused(entry, msg):
    with pytest.raises(ValueError, match=msg):
        rewards.RewardTable(_table(entry))


def test_format_tag_required(tmp_path):
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"games": {}}))
    with pytest.raises(ValueError, match="format"):
        rewards.RewardTable.load(p)


def test_addresses_and_offsets_agree():
    a = rewards.spec_from_entry({"score": ["0xD5", 0x56], "terminal": {"addr": 0xFF, "value": 1}})
    assert list(a.score_addr[:2]) == [0x55, 0x56] and a.terminal_addr == 0x7F and a.terminal_mask == 0xFF


def test_lookup_by_digest_is_exact():
    rom = bytes(range(256)) * 16
    tab = rewards.RewardTable(_table({"rom_sha256": hashlib.sha256(rom).hexdigest().upper(), "score": [0x80]}))
    assert tab.for_rom(rom) is tab.specs["g"]
    assert tab.for_rom(rom[:-1] + b"\x00") is None
