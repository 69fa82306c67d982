"""CPU checkers of the encoder-analysis path (test infrastructure, never the product).

`Oracle` binds our C restatement (oracle/vc1_oracle.c -> oracle/_oracle/libvc1oracle.so).
`Reference` binds the reference's own code compiled from its sources plus
oracle/ref_harness.cpp (oracle/_ref/libvc1ref.so). Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg use this package.
"""
from .bindings import Oracle, Reference, ref_available  # noqa: F401
