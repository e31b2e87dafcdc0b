"""CPU oracle for the SMAC pressure projection -- TEST INFRASTRUCTURE ONLY.

A C++/OpenMP restatement of the reference's pressure path (divergence,
operator assembly, the four PCG variants with the Jacobi V-cycle, velocity
correction, VoF/IBM coefficient set-up).  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` use it, and only as the checker or the CPU baseline:
the product path (``mydemcfd_b200``) never imports it.
"""
from .oracle import *  # noqa: F401,F403
