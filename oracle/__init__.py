"""ORACLE -- test infrastructure only.

CPU restatement of the reference's Newton-step hot path (Beremi/slope_stability_octave),
used exclusively as the checker by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py``.  The product package never imports this package.

Modules
-------
native      ctypes bindings of ``liboracle.so`` (C restatement, ``sg_oracle.c``) and of
            ``_ref/*.so`` (the reference's own MEX sources compiled unchanged).
octave_ref  NumPy/SciPy restatement of the Octave layer: sparse ``B``, pattern,
            scatter map, ``K_r`` values, ``F`` (``+CONSTITUTIVE_PROBLEM/CONSTITUTIVE.m``).
solvers     DFGMRES, A-orthogonalisation, direct solve (``+LINEAR_SOLVERS``).
drivers     Newton / damping / continuation (``+NEWTON``, ``+CONTINUATION``).

Parity pin: the C restatement is checked against the compiled reference kernels
(``tests/test_oracle_pin.py``) and against golden vectors made from them
(``tests/golden/make_golden.py``).
"""
