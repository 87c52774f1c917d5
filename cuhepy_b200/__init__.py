"""cuhepy_b200: the big-integer / RNS hot path of cuhepy, written for sm_100a.

- :mod:`cuhepy_b200.paillier` - Paillier and Paillier-Lookup (Montgomery CIOS
  with warp-cooperative limbs, fixed-base table products).
- :mod:`cuhepy_b200.bfv` - the BFV residue evaluator (negacyclic NTT/INTT,
  exact RNS scale-and-round, gadget key switching, packed Hamming search).
- :mod:`cuhepy_b200.hamming` - the Hamming clients with the reference API.

Kernels are reached through the C ABI in ``include/``; there is no CPU path.
"""

__version__ = "0.1.0"
__all__ = ["__version__"]
