"""B200-native reflection-tracing backend for Acoustic Agent.

The six-band listener-space path tracer (with next-event estimation to the
source), its BVH and the echogram -> band-IR synthesis run as hand-written
sm_100a kernels in ``libacoustic_rt.so``; this package is the host side:

* ``scene``      room description -> surface SoA + BVH (the reference's array contract)
* ``runtime``    resident device scenes, trace / batch / synthesis launches
* ``backend``    ``trace_energy_field`` drop-in and ``install()`` into Acoustic Agent
* ``batching``   many scenes, sources and channels in one persistent launch
* ``serving``    continuous-batching request loop with HBM admission
* ``workloads``  seeded synthetic scenes of the benchmark configurations
"""
from acoustic_agent_b200 import _lib  # noqa: F401  (fails loudly if the library is missing)
from acoustic_agent_b200.scene import SceneArrays, compile_scene  # noqa: F401

__all__ = ["SceneArrays", "compile_scene"]
__version__ = "0.1.0"
