"""CPU oracle for the gradenna FDTD hot path (test infrastructure only).

This package restates, operation for operation, the reference solver's
algorithm on the host: numpy (float32/float64) for the 2D TM and 3D Yee
steppers, the CPML tables, the port/S-parameter helpers and the Poynting
reduction, plus a multi-threaded C twin (``oracle/tm2d_ref.c``) used for the
CPU timing baseline.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import or execute anything here; the product path
(``gradenna_b200``) never does.

Parity pin: the reference's JAX path (no ``jax`` in this image) and its Rust
kernels (no ``cargo``/``rustc``) cannot run here and the reference ships no
golden vectors for ``simulate_tm`` outputs. The restatement is pinned
against the known-answer tests the reference's own test-suite holds for this
path (CPML reflection below -60 dB, late-time energy decay, Courant
stability, Re Zin = w mu0 / 4 of a free-space line port, incident wave
Vs/2, port power = Poynting flux, PEC-enclosed port |S11| = 1, 3D dipole
checks), see ``tests/test_oracle_known_answers.py``. Bit-level parity with
the reference's XLA float32 arithmetic is unpinned.
"""
