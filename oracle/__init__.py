"""CPU oracle for the halo-exchange path — TEST INFRASTRUCTURE ONLY.

A restatement of GHEX 0.4.0's pattern construction and exchange semantics in numpy and plain
Python, written independently of the product (ghex_b200/) so that it can check it:

    oracle.regular       structured::regular halo generator, make_pattern, exchange, adjoint
    oracle.cubed_sphere  cubed-sphere halo generator with tile transforms, exchange, adjoint
    oracle.unstructured  unstructured domain descriptors, make_pattern, exchange

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this package,
and only to check or to time the reference behaviour; the product never calls it.

Parity pins: the restatement is checked against the known answers of the reference's own tests
(tests/golden/, tests/test_oracle_*.py) and, where the reference's headers could be compiled
here against stub transports (oracle/ref/, built into oracle/_ref/), against the reference's own
code run on the same inputs.
"""
