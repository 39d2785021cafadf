"""Single-species solver pieces (scattering models, integrators, BCs, ICs,
moments) behind the plugin keys of dgfsStd1D."""
