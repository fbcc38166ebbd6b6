"""PyHeartSim time-stepping and electrogram hot path for NVIDIA B200 (sm_100a).

* ``pyheartsim_b200.simulation.simulation_gpu.compute`` -- drop-in for the
  reference's simulation/simulation_gpu.py::compute;
* ``pyheartsim_b200.simulation.unipolar_electrogram_gpu.compute`` -- drop-in for
  simulation/unipolar_electrogram_gpu.py::compute;
* ``pyheartsim_b200.engine.BatchedEngine`` -- many uneven instances advanced by
  one persistent launch per call;
* ``pyheartsim_b200.serving.Server`` -- continuous batching of solve requests.

All compute runs in ``libphs.so`` (C ABI: include/phs.h).
"""
__version__ = "0.1.0"
