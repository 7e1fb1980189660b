"""CPU oracle for the particle FMM (test infrastructure only).

Loaded only by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs
of bench.py.  The product library never imports this package.
"""
from .oracle import *  # noqa: F401,F403
