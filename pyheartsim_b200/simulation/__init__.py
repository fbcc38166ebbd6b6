"""Drop-in modules mirroring the reference's ``simulation`` package
(simulation/__init__.py:15-19): ``simulation_gpu``, ``unipolar_electrogram_gpu``
and the host-side ``pacing`` schedule."""
from . import pacing  # noqa: F401
from . import simulation_gpu  # noqa: F401
from . import unipolar_electrogram_gpu  # noqa: F401
