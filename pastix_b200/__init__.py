"""B200-native numerical factorization and solve backend for PaStiX.

PaStiX's host analysis stays PaStiX's C code (``pastix_b200.refhost``); numfact,
solve and refinement run on one B200 through ``libpastix_b200.so``
(``include/pastix_b200.h``, bound by ``pastix_b200.native``).  ``pastix_b200.api``
mirrors PaStiX's task API.
"""
__version__ = "0.1.0"
