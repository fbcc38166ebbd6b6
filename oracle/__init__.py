"""CPU oracle of the PyHeartSim hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker (or the timed CPU
baseline); the product package ``pyheartsim_b200`` never does.
"""
