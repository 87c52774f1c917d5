"""PaillierClient with the reference API (src/cuhepy/hamming/paillier.py:113-231).

The GPU client exchanges ciphertexts as hex strings, as the reference
pybind11 class does; this wrapper converts them back to integers.
"""

from __future__ import annotations

import json
from typing import Any

from cuhepy_b200.device import DeviceMode, resolve_device
from cuhepy_b200.hamming.base import HammingClientBase


def _load_gpu_backend() -> type[Any]:
    from cuhepy_b200.paillier.clients import PaillierGPUClient

    return PaillierGPUClient


class PaillierClient(HammingClientBase):
    def __init__(self, embed_len: int = 512, key_len: int = 1024, skip_key_gen: bool = False,
                 device: DeviceMode = "auto") -> None:
        self.embed_len = embed_len
        self.key_len = key_len
        self.chunk_len = key_len * 2
        self.chunk_num = (2 * embed_len // self.chunk_len + int((2 * embed_len) % self.chunk_len != 0)
                          if embed_len > key_len else 1)
        self.device, gpu_cls = resolve_device(device, _load_gpu_backend)
        self.client: Any = gpu_cls(embed_len=embed_len, key_len=key_len, skip_key_gen=skip_key_gen)

    @staticmethod
    def has_gpu() -> bool:
        try:
            _load_gpu_backend()(skip_key_gen=True)
            return True
        except Exception:
            return False

    @staticmethod
    def _cipher_to_int(value: Any) -> int:
        if isinstance(value, bytes):
            return int.from_bytes(value, byteorder="little")
        if isinstance(value, str):
            return int(value, 16)
        return int(value)

    @staticmethod
    def _cipher_to_hex(value: int | bytes) -> str:
        if isinstance(value, bytes):
            return format(int.from_bytes(value, byteorder="little"), "x")
        return format(int(value), "x")

    def encrypt_vec_one(self, embd: list[int]) -> list[int]:
        if len(embd) != self.embed_len:
            raise ValueError(f"Embedding length {len(embd)} does not match expected {self.embed_len}")
        return [self._cipher_to_int(c) for c in self.client.encrypt([embd])[0]]

    def encrypt_vec_batch(self, embds: list[list[int]]) -> list[list[int]]:
        return [[self._cipher_to_int(c) for c in row] for row in self.client.encrypt(embds)]

    def decode_hamming_client_one(self, cipher: list[int | bytes]) -> int:
        return int(self.client.decode_hamming_client([[self._cipher_to_hex(v) for v in cipher]])[0])

    def decode_hamming_client_batch(self, ciphers: list[list[int | bytes]]) -> list[int]:
        return [int(v) for v in self.client.decode_hamming_client(
            [[self._cipher_to_hex(e) for e in cipher] for cipher in ciphers])]

    def stringify_pk(self) -> str:
        return self.client.stringify_pk()

    def stringify_sk(self) -> str:
        return self.client.stringify_sk()

    def stringify_config(self) -> str:
        return self.client.stringify_config()

    def load_stringified_keys(self, pk: str, sk: str) -> None:
        self.client.load_stringified_keys(pk, sk)

    def load_config(self, config: dict) -> None:
        self.client.load_config({k: v for k, v in config.items() if k != "device"})
        self.embed_len = config["embed_len"]
        self.key_len = config["key_len"]
        self.chunk_len = self.key_len * 2
        self.chunk_num = (2 * self.embed_len // self.chunk_len + int((2 * self.embed_len) % self.chunk_len != 0)
                          if self.embed_len > self.key_len else 1)

    def encode_hamming_server(self, ct1: list[int | bytes], ct2: list[int | bytes]) -> list[int]:
        if len(ct1) != len(ct2):
            raise ValueError("ct1 and ct2 must have the same length")
        pk = json.loads(self.stringify_pk())
        result = type(self.client).encode_hamming_server(
            [self._cipher_to_hex(c) for c in ct1], [self._cipher_to_hex(c) for c in ct2],
            {"n_squared": format(int(pk["n_squared"]), "x")})
        return [self._cipher_to_int(c) for c in result]
