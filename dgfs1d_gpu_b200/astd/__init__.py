"""Penalised IMEX solver pieces behind the plugin keys of dgfsABstd1D."""
