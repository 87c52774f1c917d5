"""BFV evaluator on the B200.

:mod:`._bfv_rns` is a drop-in for the reference's native module of the same
name (ABI 4): residue rings (Q a product of NTT primes, ``residue=True``) and
native rings with any odd modulus q up to 512 bits (``residue=False``, the
reference's default prime-q client), every function of the reference module
plus resident-index search, batched NTTs and client-side encryption.  The
reference's own Python layer (``BFVNativeServer``, ``BFVRNSArithmetic``)
runs on it unchanged.  :mod:`.layout` holds the packed Hamming layout and
wire helpers, :mod:`.client` the batched client-side encryption.
"""
