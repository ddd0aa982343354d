"""The oracle of the FFT3D filtering core — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker; the product
(``neo_fft3d_b200``) never imports it.

* :mod:`oracle.restate` — CPU restatement of the reference pipeline
  (``fft3d_oracle.cpp``): float mode reproduces the reference's C path (opt=1)
  bit for bit given the same FFT; double mode is the FP64 truth.
* :mod:`oracle.reference` — the UNMODIFIED reference plugin, compiled from its
  own sources by ``oracle/Makefile`` into ``oracle/_ref`` and run through the
  headless VapourSynth host behind the FFTW-API shim (``fftw_shim.cpp``).
"""
