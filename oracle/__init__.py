"""CPU oracle for the Lax-Friedrichs hot path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker.  The product path
(``mpd-plasma-dynamics_b200/``) never imports, links or calls it.
"""
