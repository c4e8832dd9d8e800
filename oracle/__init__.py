"""CPU oracle for the matrix-free Rydberg ED path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product package imports this package.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it,
always as the checker (or the timed CPU baseline), never as the thing
measured or shipped.

``ref.py`` restates the reference algorithms in numpy (each function cites
the reference file:line it follows); ``el_oracle.c`` restates the full-basis
H-apply and the KPM recurrence in C with OpenMP for the timed CPU baseline.
The restatement is pinned against golden vectors produced by the reference
itself (``tests/golden/make_golden.py``).
"""
