"""TEST INFRASTRUCTURE ONLY: the CPU oracle (C++ restatement of the
reference's time step) and its ctypes wrapper.  Imported by the tests, the
smoke check and the CPU-baseline leg of bench.py, never by the product."""
