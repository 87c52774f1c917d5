"""Encrypted Hamming-distance clients with the reference API, on the B200."""
