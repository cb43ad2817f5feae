"""fmm_gen_b200: B200-native generated fast matrix multiplication (FMM).

Layers:
  algebra   -- coefficient grammar, [U,V,W] files, Kronecker composition, fringe split
  alg_dic   -- algorithm name table
  control   -- the generator CLI (N alg L ... pack_type gen_path)
  runtime   -- ctypes binding of the sm_100a library (include/fmm_b200.h)
"""
from . import algebra  # noqa: F401
from .alg_dic import alg_dic  # noqa: F401

__all__ = ["algebra", "alg_dic"]
