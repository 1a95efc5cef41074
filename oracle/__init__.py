"""CPU oracle of the Band path -- TEST INFRASTRUCTURE ONLY.

Restatements of the reference algorithm (yumiaoyi-o/AOSpectrum) used as the
checker by ``tests/``, by ``__graft_entry__.smoke()`` and by the CPU
baseline legs of ``bench.py``.  Nothing in ``aospectrum_b200`` imports this
package: the product path runs on the GPU through libaospectrum_b200.so and
fails loudly without it.

Modules:
  bloch_ref   numpy restatement of BlochPattern.from_bundle and
              BlochWorkspace.update (src/aospectrum/sparse.py:25-245)
  bloch_c     ctypes wrapper of bloch_ref.c, the same Bloch sum in plain C
  ciss_ref    numpy/scipy restatement of CudssCissSolver.solve_interval
              (src/aospectrum/ciss.py:81-391) with CPU shifted solves
  dense_ref   FP64 dense generalized eigenvalues of H(k), S(k)

Pinning: bloch_ref and ciss_ref are checked against golden vectors that
tests/golden/make_golden.py produced by importing the reference's own
Python package (the reference ships no tests or fixtures of its own).
"""
