"""CPU oracle for the lens_sensor FDTD time-stepping path.

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, by ``__graft_entry__.smoke()``
and by ``bench.py``'s CPU-baseline leg, and by nothing else.  The product package
``lens_sensor_b200`` never imports, links or executes anything from here.
"""
