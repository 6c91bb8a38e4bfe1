"""Parity oracle for the SFR3D linear-solve path (test infrastructure only).

``oracle.oracle`` wraps two CPU libraries:

* ``liboracle.so`` -- the C restatement in ``sfr3d_oracle.c``;
* ``_ref/libsfr3d_ref.so`` -- the reference's own solver sources compiled
  by ``oracle/Makefile`` plus ``ref_harness.c`` (present only where the
  reference checkout was available at build time, or where the built file
  was carried along).

Only tests, the smoke check and bench.py's CPU-baseline leg may use them.
"""
