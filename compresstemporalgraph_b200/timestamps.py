"""Timestamp bucketing of the compressed format (TimestampComparerAggregator.java:8-23).

The stored delta between consecutive timestamps of a list is ``b // f - a // f`` for an
aggregation factor ``f``; decoding restores ``previous + f * delta``, and the stream header holds
the minimum timestamp rounded down to a multiple of ``f``.  The reference runner and every GPU
kernel use ``f = 1`` (BaselineRunner.java:17), which is what the engine decodes; these helpers
keep the general definitions for tools that build or inspect aggregated streams.
"""
from __future__ import annotations


def _check(factor: int) -> None:
    if factor < 1:
        raise ValueError("factor must be positive")


def _floordiv(a: int, f: int) -> int:
    # Java's integer division truncates toward zero.
    q = abs(a) // f
    return q if a >= 0 else -q


def timestamps_difference(first: int, second: int, factor: int) -> int:
    _check(factor)
    return _floordiv(second, factor) - _floordiv(first, factor)


def reverse(previous: int, difference: int, factor: int) -> int:
    _check(factor)
    return previous + factor * difference


def aggregate_min_timestamp(minimum: int, factor: int) -> int:
    _check(factor)
    return _floordiv(minimum, factor) * factor
