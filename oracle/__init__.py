"""CPU FP64 oracle for OpenParEM3D's per-frequency FEM solve stage.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``openparem_b200``) may
import, call or link anything in this package.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` use it, and there only as the checker or as the timed
CPU restatement of the reference path.

What it restates (reference files cited by path inside the OpenParEM tree):

* weak form and boundary terms: doc/OpenParEM3D_Theory_Methodology_Accuracy.tex:82-201
* operator assembly:             src/OpenParEM3D/fem3D.cpp:103-190 (build_A)
* non-driven port 2D ABC:        src/OpenParEM3D/port.cpp:5783-5875 (Port::addPortIntegrators)
* impedance / radiation term:    src/OpenParEM3D/port.cpp:1009-1041 (Boundary::addImpedanceIntegrator)
* PEC elimination:               src/OpenParEM3D/fem3D.cpp:80-99, solveComplexLinearSystem.c:61-65
* driven-port Dirichlet lifting: src/OpenParEM3D/solveComplexLinearSystem.c:114-129
* H projection P h = j Q e:      src/OpenParEM3D/fem3D.cpp:192-225, 610-648
* port overlaps C+/C-:           src/OpenParEM3D/port.cpp:3463-3489, 3524-3568
* S-matrix solve:                src/OpenParEM3D/port.cpp:7499-7606
* forced reciprocity:            src/OpenParEM3D/results.cpp:401-418
* material models:               src/OpenParEMCommon/OpenParEMmaterials.cpp:600-883

The Nedelec (first kind, order p) space is MFEM's ``ND_FECollection(p,3)``
space; the basis inside it is this project's own (moment degrees of freedom
on globally sorted vertices), so element matrices are compared with the GPU
path, not with MFEM.  Parity against the reference itself is pinned at the
S-parameter level by the WR90 regression cases (tests/golden/).
"""
