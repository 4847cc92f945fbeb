"""CPU oracle for the TholeDipoleForce hot path.  Test infrastructure only:
the parity tests, the smoke check and bench.py's CPU-baseline leg call it as
the checker; the shipped library never imports it."""
