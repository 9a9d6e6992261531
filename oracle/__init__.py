"""CPU oracle for the RNS walk path: TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU, what the reference computes on the walk
path (reference python/dreams_rns/runner.py, cmf_walk.py).  It is the checker
for the CUDA library, never part of it: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline leg and its
``--impl reference`` arm) may import or run anything under ``oracle/``.  The
product package ``dreams_rns`` never imports it and has no CPU fallback.

Modules
-------
``walk_np``  numpy restatement of the reference walk, CRT and delta functions,
             one function per reference function (file:line cited on each).
             Vectorised over the K primes per step exactly like the reference,
             so its speed is representative of the reference's own CPU path.
``walk_c``   ctypes wrapper around ``walk_oracle.c``: the same per-step
             semantics in plain C, fast enough for parity sweeps over
             thousands of walks.  Built by ``oracle/build.py`` into
             ``oracle/_build/``.

Pinning: ``tests/test_oracle_golden.py`` checks both restatements against
``tests/golden/reference_golden.json``, which ``tests/golden/make_golden.py``
produced by importing and running the reference package itself.
"""
