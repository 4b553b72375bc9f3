"""CPU oracle for the SOLWEIG radiation chain -- TEST INFRASTRUCTURE ONLY.

This package is a CPU restatement of the reference implementation
(Synn-Arch/Solweig_Project, ``solweig_gpu``) of the path the CUDA library
accelerates: the SVF patch sweep, the wall-height sun march, the ground view
factor walk, the short/long-wave fluxes, Tmrt and UTCI.  Planes are numpy
float32 arrays evaluated in the reference's operation order; 0-dim scalars are
evaluated with 0-dim torch CPU tensors where the reference does so, so that
their float32 rounding (and the trigonometric calls that feed the march step
tables) follow the reference bit for bit.

It is the checker: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline arm of ``bench.py`` import it.  The product
(``solweig_project_b200``) never imports or calls anything here.

Parity of this oracle is pinned against golden fixtures produced by running
the reference itself (``tests/golden/make_golden.py``).
"""
