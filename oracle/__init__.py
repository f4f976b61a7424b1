"""CPU oracle for the TopOpt-SLP-3D equilibrium-solve path.

TEST INFRASTRUCTURE ONLY.  This package is a plain NumPy/SciPy (and C, see
``kelem_omp.c``) restatement of the reference MATLAB functions on the hot path.
It exists so that ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` can check and time
the CUDA library against the reference algorithm.  The product path (the
``tosp`` C-ABI library and its Python binding) never imports, links or calls
anything in here.

Every function cites the reference file and line range it follows
(paths relative to the reference project root, ``Implementation/`` written as
``I/``).  Indices are 0-based here; the reference is 1-based.

Parity pins: the reference is MATLAB-only and cannot run on this machine, and
it ships no stored outputs.  The oracle is pinned by
  * the closed-form hex8 stiffness of ``I/ElemStiffMatrix.m`` (golden values
    produced by evaluating that file's assignment statements, see
    ``tests/golden/make_golden.py``),
  * the ``freedofs`` / ``f`` arrays stored in the reference's own problem
    fixtures (``I/Tests/*.mat``), reproduced from their ``supp``/``loads`` rows,
  * the reference's internal cross-implementations (matrix-free ``KelemProd``
    versus assembled ``GlobalStiffMatrix``; ``SolveMG`` versus a direct solve).
"""
