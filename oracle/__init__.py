"""The oracle: test infrastructure only (never imported by the product).

C restatement of the reference's photon-propagation path (lmc_oracle.c), the
MIEV0 restatement (miev0.c), the Philox replay seam for the reference
(replay_rng.cpp) and the recipe that compiles the reference into oracle/_ref
(Makefile).  Python access: ``oracle.pyoracle``.
"""
