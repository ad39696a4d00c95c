"""Test infrastructure: CPU oracles for the compact neighbour search.

Only ``tests/``, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline / reference arms may
import this package, and only as the checker.  The product package never imports it.
"""
