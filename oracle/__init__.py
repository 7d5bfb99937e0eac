"""TEST INFRASTRUCTURE ONLY: the oracles the tests check the device against.

  refharness   the reference renderer itself (oracle/_ref, built from the
               reference's sources by oracle/Makefile)
  restatement  the C restatement of the reference's hot path
               (lambda_oracle.c, built into oracle/_build/liboracle.so)

Nothing in the product imports this package.
"""
