"""PaillierLookupClient with the reference API (src/cuhepy/hamming/paillier_lookup.py).

Dispatch, argument checks, weak-alpha policy and pickling follow the
reference class (paillier_lookup.py:245-425); the arithmetic runs in
:class:`cuhepy_b200.paillier.clients.PaillierGPULookupClient`.
"""

from __future__ import annotations

import json
import warnings
from typing import Any

from cuhepy_b200.device import DeviceMode, resolve_device
from cuhepy_b200.hamming.base import HammingClientBase
from cuhepy_b200.paillier.lookup import DEFAULT_ALPHA_LEN, MIN_ALPHA_LEN


def _reject_weak_alpha(alpha_len: int, allow_weak_alpha: bool) -> None:
    if alpha_len < MIN_ALPHA_LEN and not allow_weak_alpha:
        raise ValueError(
            f"alpha_len={alpha_len} is insecure: the secret exponent is recoverable "
            f"from the public key in ~2**{alpha_len // 2} operations. Use "
            f"alpha_len >= {MIN_ALPHA_LEN} (default {DEFAULT_ALPHA_LEN}), or pass "
            f"allow_weak_alpha=True for cryptanalysis work."
        )


def _warn_weak_alpha(alpha_len: int) -> None:
    if alpha_len < MIN_ALPHA_LEN:
        warnings.warn(
            f"Loaded a Paillier-Lookup key with alpha_len={alpha_len}; its secret "
            f"exponent is recoverable from the public key. Regenerate with "
            f"alpha_len >= {MIN_ALPHA_LEN}.",
            RuntimeWarning,
            stacklevel=3,
        )


def _load_gpu_backend() -> type[Any]:
    from cuhepy_b200.paillier.clients import PaillierGPULookupClient

    return PaillierGPULookupClient


def _layout(embed_len: int, key_len: int) -> tuple[int, int]:
    chunk_len = key_len * 2
    chunk_num = 2 * embed_len // chunk_len + int((2 * embed_len) % chunk_len != 0) if embed_len > key_len else 1
    return chunk_len, chunk_num


class PaillierLookupClient(HammingClientBase):
    def __init__(self, embed_len: int = 512, key_len: int = 1024, alpha_len: int = DEFAULT_ALPHA_LEN,
                 skip_key_gen: bool = False, device: DeviceMode = "auto", allow_weak_alpha: bool = False) -> None:
        if not skip_key_gen:
            _reject_weak_alpha(alpha_len, allow_weak_alpha)
        self.alpha_len = alpha_len
        self.key_len = key_len
        self.embed_len = embed_len
        self.chunk_len, self.chunk_num = _layout(embed_len, key_len)
        self.device, gpu_cls = resolve_device(device, _load_gpu_backend)
        self.client: Any = gpu_cls(embed_len=embed_len, key_len=key_len, alpha_len=alpha_len,
                                   skip_key_gen=skip_key_gen)

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
        return int(value)

    def encrypt_vec_one(self, embd: list[int]) -> list[int]:
        if len(embd) != self.embed_len:
            raise ValueError(f"Embedding length {len(embd)} does not match expected {self.embed_len}")
        return [self._cipher_to_int(c) for c in self.client.encrypt([embd])[0]]

    def encrypt_vec_batch(self, embds: list[list[int]]) -> list[list[int]]:
        return [[self._cipher_to_int(c) for c in row] for row in self.client.encrypt(embds)]

    def decode_hamming_client_one(self, cipher: list[int | bytes]) -> int:
        return int(self.client.decode_hamming_client([[self._cipher_to_int(v) for v in cipher]])[0])

    def decode_hamming_client_batch(self, ciphers: list[list[int | bytes]]) -> list[int]:
        normalized = [[self._cipher_to_int(v) for v in cipher] for cipher in ciphers]
        return [int(v) for v in self.client.decode_hamming_client(normalized)]

    def stringify_pk(self) -> str:
        return self.client.stringify_pk()

    def stringify_sk(self) -> str:
        return self.client.stringify_sk()

    def stringify_config(self) -> str:
        return self.client.stringify_config()

    def load_stringified_keys(self, pk: str, sk: str) -> None:
        self.client.load_stringified_keys(pk, sk)

    def load_config(self, config: dict, precomputed_tables: dict | None = None) -> None:
        sanitized = {k: v for k, v in config.items() if k != "device"}
        self.client.load_config(sanitized, precomputed_tables)
        self.embed_len = config["embed_len"]
        self.key_len = config["key_len"]
        self.alpha_len = config.get("alpha_len", self.alpha_len)
        _warn_weak_alpha(self.alpha_len)
        self.chunk_len, self.chunk_num = _layout(self.embed_len, self.key_len)

    def encode_hamming_server(self, ct1: list[int | bytes], ct2: list[int | bytes]) -> list[int]:
        if len(ct1) != len(ct2):
            raise ValueError("ct1 and ct2 must have the same length")
        result = type(self.client).encode_hamming_server(
            [self._cipher_to_int(c) for c in ct1], [self._cipher_to_int(c) for c in ct2],
            json.loads(self.stringify_pk()))
        return [self._cipher_to_int(c) for c in result]

    def dump_tables(self) -> dict:
        return self.client.dump_tables()

    def __getstate__(self) -> dict:
        state = {"embed_len": self.embed_len, "key_len": self.key_len, "alpha_len": self.alpha_len,
                 "pk": self.stringify_pk(), "sk": self.stringify_sk(),
                 "config": json.loads(self.stringify_config())}
        tables = self.dump_tables()
        if tables:
            state["tables"] = tables
        return state

    def __setstate__(self, state: dict) -> None:
        self.embed_len = state["embed_len"]
        self.key_len = state["key_len"]
        self.alpha_len = state["alpha_len"]
        self.chunk_len, self.chunk_num = _layout(self.embed_len, self.key_len)
        self.device, gpu_cls = resolve_device("auto", _load_gpu_backend)
        self.client = gpu_cls(embed_len=self.embed_len, key_len=self.key_len, alpha_len=self.alpha_len,
                              skip_key_gen=True)
        self.client.load_stringified_keys(state["pk"], state["sk"])
        self.load_config(state["config"], precomputed_tables=state.get("tables"))
