"""Paillier and Paillier-Lookup on the B200: reference-compatible static APIs
(:mod:`.scheme`, :mod:`.lookup`), device contexts (:mod:`.gpu`) and the GPU
client classes (:mod:`.clients`)."""
