"""Autotuner host logic (no GPU): the cache key separates library builds whose kernels have
different residencies, and a cached shape is clamped to the current residencies."""
import numpy as np

from cumayo_b200 import autotune as AT


def _items():
    # op in bits 30-31, set index in 28-29 (the queue's item layout); any values give a signature
    return (np.arange(64, dtype=np.uint32) % 12) << 28


def test_cache_key_includes_residency():
    per_a = {(1, 0): 3, (1, 1): 2, (5, 2): 4}
    per_b = dict(per_a)
    per_b[(5, 2)] = 3
    ka = AT.cache_key("B200", 148, per_a, _items())
    kb = AT.cache_key("B200", 148, per_b, _items())
    assert ka != kb
    assert ka == AT.cache_key("B200", 148, dict(reversed(list(per_a.items()))), _items())  # order-free
    assert ka != AT.cache_key("B200", 132, per_a, _items())


def test_clamp_shape():
    per = {(1, 0): 3, (5, 2): 2}
    assert AT.clamp_shape({(1, 0): 5, (5, 2): 2}, per) == {(1, 0): 3, (5, 2): 2}
    assert AT.clamp_shape({(1, 0): 0, (5, 2): 1}, per) == {(1, 0): 1, (5, 2): 1}
