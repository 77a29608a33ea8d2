"""Test infrastructure: the CPU oracle of the MPM substep.

`oracle.restated` runs the C restatement (oracle/*.c, FP32 and FP64) through ctypes;
`oracle.reference` runs the reference's own OpenMP/sequential path, compiled from its
sources by oracle/build_ref.sh, as a subprocess.  Only tests, the smoke check and the
benchmark's CPU-baseline leg use this package; the product never does.
"""
