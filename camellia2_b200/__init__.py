"""camellia2_b200 — B200-native DPG per-cell assembly (Camellia's
BF::localStiffnessMatrixAndRHS + CondensedDofInterpreter Schur complement)."""
from . import abi, formulation, mesh  # noqa: F401
