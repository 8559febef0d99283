"""Sharding of independent work over ranks (piernik_b200/shard.py), host
side: block lists balanced by cell count and instance ranges, deterministic
and complete."""
import pytest

from piernik_b200.shard import balance, instance_ranges


def test_balance_covers_every_block_once():
    cells = [16 ** 3, 64 ** 3, 24 * 32 * 48, 48 ** 3, 16 * 16 * 64, 32 ** 3, 64 * 48 * 16]
    for world in (1, 2, 3, 4):
        parts = balance(cells, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(cells)))
        assert all(p == sorted(p) for p in parts)
        loads = [sum(cells[i] for i in p) for p in parts]
        # greedy largest-first: no rank exceeds the lightest by more than the largest block
        assert max(loads) - min(loads) <= max(cells)
        assert balance(cells, world) == parts          # the same on every rank


def test_instance_ranges():
    assert instance_ranges(64, 8) == [(8 * r, 8 * r + 8) for r in range(8)]
    assert instance_ranges(10, 3) == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError):
        instance_ranges(2, 3)
