"""CPU oracle of TomoSTAR's forward path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this package,
as the checker and the timed CPU baseline. The product package ``tomostar_b200`` never does.
"""
