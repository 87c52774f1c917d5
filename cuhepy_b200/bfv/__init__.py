"""BFV residue evaluator on the B200.

:mod:`._bfv_rns` is a drop-in for the reference's native module of the same
name (ABI 4) for residue rings; :mod:`.native` mirrors the reference's
``BFVNativeServer`` wire framing on top of it.
"""
