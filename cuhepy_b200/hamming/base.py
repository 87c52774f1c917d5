"""HammingClientBase (src/cuhepy/hamming/base.py)."""

from abc import ABC, abstractmethod


class HammingClientBase(ABC):
    @abstractmethod
    def encrypt_vec_one(self, embd: list[int]) -> list[int]: ...

    @abstractmethod
    def encrypt_vec_batch(self, embds: list[list[int]]) -> list[list[int]]: ...

    @abstractmethod
    def decode_hamming_client_one(self, cipher: list[int | bytes]) -> int: ...

    @abstractmethod
    def decode_hamming_client_batch(self, ciphers: list[list[int | bytes]]) -> list[int]: ...
