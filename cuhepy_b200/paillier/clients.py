"""B200 replacements of the reference's pybind11 GPU client classes.

``PaillierGPULookupClient`` mirrors the method set of
src/cuhepy/paillier/_lookup_gpu_ext/paillier_GPU_lookup_client.cu:2673-2722 and
``PaillierGPUClient`` that of src/cuhepy/paillier/_gpu_ext/paillier_GPU_client.cu:
1136-1166, with the same argument meanings, return types (lookup: ints, plain:
hex strings) and error behaviour (``RuntimeError`` on missing keys, shape or
binary-value violations).  Unlike the reference binaries, which are compiled
for one KEY_BITS, any key_len up to ``KEY_BITS`` runs at run time.
"""

from __future__ import annotations

import json
import math
import secrets
from collections.abc import Sequence

import numpy as np

from cuhepy_b200.paillier.gpu import NOISE_MULTIPLES, device_for
from cuhepy_b200.paillier.lookup import DEFAULT_ALPHA_LEN, PaillierLookup, message_chunks_for
from cuhepy_b200.paillier.scheme import Paillier

KEY_BITS = 2048  # largest prime size (n^2 of 8192 bits) the kernels are compiled for


def chunk_layout(embed_len: int, key_len: int) -> tuple[int, int]:
    """(chunk_len, chunk_num) as in hamming/paillier_lookup.py:73-77."""
    chunk_len = key_len * 2
    if embed_len > key_len:
        chunk_num = 2 * embed_len // chunk_len + int((2 * embed_len) % chunk_len != 0)
    else:
        chunk_num = 1
    return chunk_len, chunk_num


def _bits_array(embeddings: Sequence[Sequence[int]], embed_len: int) -> np.ndarray:
    for row in embeddings:
        if len(row) != embed_len:
            raise RuntimeError("encrypt: each embedding must have length == embed_len")
    arr = np.asarray([list(row) for row in embeddings], dtype=np.int64).reshape(len(embeddings), embed_len)
    if arr.size and ((arr != 0) & (arr != 1)).any():
        raise RuntimeError("encrypt: embeddings must be binary 0/1")
    return np.ascontiguousarray(arr, dtype=np.uint8)


def _chunk_plaintexts(bits: np.ndarray, chunk_len: int, chunk_num: int, words: int) -> np.ndarray:
    """Hamming plaintexts [vectors * chunk_num, words] (little-endian u32) of
    a [vectors, embed_len] bit matrix: bit j at padded position 2j + 1 of the
    string "0 b_0 0 b_1 ...", cut into chunk_len-bit chunks, each read most
    significant bit first (hamming/paillier.py:76-88), vectorised."""
    vectors, embed = bits.shape
    padded = np.zeros((vectors, 2 * embed), dtype=np.uint8)
    padded[:, 1::2] = bits
    # chunk c is the substring [c chunk_len, (c + 1) chunk_len) of the padded
    # string (the last one possibly shorter), right-aligned in chunk_len bits
    chunks = np.zeros((vectors, chunk_num, chunk_len), dtype=np.uint8)
    for c in range(chunk_num):
        piece = padded[:, c * chunk_len:(c + 1) * chunk_len]
        chunks[:, c, chunk_len - piece.shape[1]:] = piece
    big = np.packbits(chunks.reshape(vectors * chunk_num, chunk_len), axis=1, bitorder="big")  # MSB first
    out = np.zeros((vectors * chunk_num, 4 * words), dtype=np.uint8)
    out[:, :big.shape[1]] = big[:, ::-1]
    return out.view(np.uint32)


def _as_int(value) -> int:
    if isinstance(value, bytes):
        return int.from_bytes(value, "little")
    if isinstance(value, str):
        text = value.strip()
        return int(text, 16) if text.lower().startswith("0x") else int(text)
    return int(value)


def _ciphertexts(values, n_squared: int) -> list[int]:
    """Ciphertext operands as the reference's bigint_to_mem takes them
    (paillier_GPU_lookup_client.cu:525-533): any value of the context's
    width, reduced mod n^2 here (every kernel result depends on c mod n^2
    only); wider values are rejected with the reference's message."""
    limit = 1 << (32 * max(1, (n_squared.bit_length() + 31) // 32))
    out = []
    for v in values:
        c = _as_int(v)
        if not 0 <= c < limit:
            raise RuntimeError("bigint_to_mem: value does not fit in mem_t")
        out.append(c % n_squared)
    return out


def _g_table_from_py(obj, message_chunks: int) -> dict[int, list[int]]:
    """g_table_from_py (paillier_GPU_lookup_client.cu:1377-1426): a dict keyed
    by row number (int or str) or a sequence of exactly message_chunks rows,
    each of 256 entries; rows past message_chunks in a dict are ignored."""
    if obj is None:
        return {}

    def row(values) -> list[int]:
        values = list(values)
        if len(values) != 256:
            raise RuntimeError("g_table row length mismatch")
        return [_as_int(v) for v in values]

    if isinstance(obj, dict):
        out = {}
        for i in range(message_chunks):
            if i in obj:
                out[i] = row(obj[i])
            elif str(i) in obj:
                out[i] = row(obj[str(i)])
            else:
                raise RuntimeError("g_table missing row")
        return out
    if isinstance(obj, Sequence) and not isinstance(obj, (str, bytes)):
        if len(obj) != message_chunks:
            raise RuntimeError("g_table outer length mismatch")
        return {i: row(obj[i]) for i in range(message_chunks)}
    raise RuntimeError("g_table must be dict or sequence")


class PaillierGPULookupClient:
    """Paillier-Lookup client whose arithmetic runs on the B200."""

    @staticmethod
    def max_key_len() -> int:
        return KEY_BITS

    def __init__(self, embed_len: int = 512, key_len: int = 1024, alpha_len: int = DEFAULT_ALPHA_LEN,
                 skip_key_gen: bool = False) -> None:
        if key_len > KEY_BITS:
            raise RuntimeError(f"PaillierGPULookupClient: key_len={key_len} exceeds KEY_BITS={KEY_BITS}")
        self._embed_len = int(embed_len)
        self._key_len = int(key_len)
        self.alpha_len = int(alpha_len)
        self._chunk_len, self._chunk_num = chunk_layout(self._embed_len, self._key_len)
        self.keys: dict | None = None
        self.message_chunks = 0
        if not skip_key_gen:
            self.keys = PaillierLookup.key_gen(self._key_len, self.alpha_len)
            self.message_chunks = self.keys["message_chunks"]
            self._install_tables()
        device_for_probe()

    # -- properties -------------------------------------------------------
    embed_len = property(lambda self: self._embed_len)
    key_len = property(lambda self: self._key_len)
    chunk_len = property(lambda self: self._chunk_len)
    chunk_num = property(lambda self: self._chunk_num)

    def _need_keys(self, what: str) -> dict:
        if self.keys is None:
            raise RuntimeError(f"{what}: keys not initialized")
        return self.keys

    def _ctx(self):
        keys = self._need_keys("device")
        return device_for(int(keys["pk"]["n"]), (int(keys["sk"]["a"]), int(keys["sk"]["g_a_inv"])),
                          phi=keys["sk"].get("phi"))

    def _table_fingerprint(self) -> tuple:
        keys = self._need_keys("tables")
        rows, noise = keys.get("g_table") or {}, keys.get("noise_table") or []
        if not rows or not noise:
            return ()
        last = rows[self.message_chunks - 1]
        return (self.message_chunks, len(noise), int(rows[0][1]), int(last[1]), int(last[255]),
                int(noise[0]), int(noise[-1]))

    def _install_tables(self) -> None:
        """Put this client's tables on its device context.  Contexts are
        shared by key, so the installed tables carry a fingerprint and a
        client whose tables differ reinstalls its own before encrypting."""
        keys = self._need_keys("tables")
        ctx = self._ctx()
        rows = [keys["g_table"][i] for i in range(self.message_chunks)]
        if rows and keys["noise_table"]:
            ctx.set_tables(rows, keys["noise_table"])
            ctx._client_tables = self._table_fingerprint()

    def _ensure_tables(self) -> None:
        keys = self._need_keys("tables")
        if not keys.get("g_table") or not keys.get("noise_table"):
            chunks = self.message_chunks or message_chunks_for(self._key_len)
            self.message_chunks = chunks
            keys["g_table"] = PaillierLookup.precompute_g_table(keys["pk"]["g"], keys["pk"]["n"], self._key_len)
            keys["noise_table"] = PaillierLookup.precompute_noise_table(keys["pk"]["g"], keys["pk"]["n"])
            keys["message_chunks"] = chunks
        ctx = self._ctx()
        if getattr(ctx, "_client_tables", None) != self._table_fingerprint():
            self._install_tables()

    # -- encryption -------------------------------------------------------
    def _noise_indices(self, count: int) -> np.ndarray:
        size = len(self._need_keys("noise")["noise_table"])
        draws = [secrets.randbelow(size) for _ in range(count * NOISE_MULTIPLES)]
        return np.asarray(draws, dtype=np.uint8).reshape(count, NOISE_MULTIPLES)

    def encrypt(self, embeddings: Sequence[Sequence[int]], noise_index: np.ndarray | None = None) -> list[list[int]]:
        self._need_keys("encrypt")
        self._ensure_tables()
        if len(embeddings) == 0:
            return []
        bits = _bits_array(embeddings, self._embed_len)
        if noise_index is None:
            noise_index = self._noise_indices(len(embeddings) * self._chunk_num)
        return self._ctx().lookup_encrypt_bits(bits, self._chunk_len, self._chunk_num, noise_index)

    def encrypt_cts(self, plaintexts: Sequence[int], noise_index: np.ndarray | None = None) -> list[int]:
        keys = self._need_keys("encrypt_cts")
        self._ensure_tables()
        values = [_as_int(v) for v in plaintexts]
        n = int(keys["pk"]["n"])
        if any(not 0 <= v < n for v in values):
            raise RuntimeError("encrypt_cts: plaintext out of range [0, n)")
        if noise_index is None:
            noise_index = self._noise_indices(len(values))
        return self._ctx().lookup_encrypt_ints(values, noise_index)

    def decrypt_cts(self, ciphers: Sequence[int]) -> list[int]:
        keys = self._need_keys("decrypt_cts")
        return self._ctx().decrypt(_ciphertexts(ciphers, int(keys["pk"]["n_squared"])))

    def decrypt_then_reencrypt(self, ciphers: Sequence[int], key_a: dict, key_b: dict) -> list[int]:
        """paillier_GPU_lookup_client.cu:2134-2286: decrypt under key_a, re-encrypt under key_b."""
        pk_a, sk_a = key_a.get("pk", key_a), key_a.get("sk", key_a)
        pk_b = key_b.get("pk", key_b)
        plain = device_for(int(pk_a["n"]), (int(sk_a["a"]), int(sk_a["g_a_inv"])), phi=sk_a.get("phi")).decrypt(
            [_as_int(c) for c in ciphers])
        n_b = int(pk_b["n"])
        chunks = int(key_b.get("message_chunks") or message_chunks_for((n_b.bit_length() + 1) // 2))
        g_table = key_b.get("g_table") or PaillierLookup.precompute_g_table(int(pk_b["g"]), n_b, chunks * 4)
        noise = key_b.get("noise_table") or PaillierLookup.precompute_noise_table(int(pk_b["g"]), n_b)
        idx = np.asarray([secrets.randbelow(len(noise)) for _ in range(len(plain) * NOISE_MULTIPLES)],
                         dtype=np.uint8).reshape(len(plain), NOISE_MULTIPLES)
        return PaillierLookup.encrypt_batch([m % n_b for m in plain], pk_b, g_table, noise, chunks, noise_index=idx)

    # -- homomorphic evaluation and decoding ---------------------------------
    def encode_hamming_client(self, ct1: Sequence[int], ct2: Sequence[int]) -> list[int]:
        keys = self._need_keys("encode_hamming_client")
        if len(ct1) != len(ct2):
            raise RuntimeError("encode_hamming_client: ct1 and ct2 must have the same length")
        return device_for(int(keys["pk"]["n"])).mulmod([_as_int(c) for c in ct1], [_as_int(c) for c in ct2])

    @staticmethod
    def encode_hamming_server(ct1: Sequence[int], ct2: Sequence[int], pk: dict) -> list[int]:
        if len(ct1) != len(ct2):
            raise RuntimeError("encode_hamming_server: ct1 and ct2 must have the same length")
        pk = pk.get("pk", pk)
        if "n_squared" not in pk:
            raise RuntimeError("encode_hamming_server: pk must contain n_squared")
        n = int(pk["n"]) if "n" in pk else math.isqrt(_as_int(pk["n_squared"]))
        return device_for(n).mulmod([_as_int(c) for c in ct1], [_as_int(c) for c in ct2])

    def decode_hamming_client(self, ciphers_batch: Sequence[Sequence[int]]) -> list[int]:
        keys = self._need_keys("decode_hamming_client")
        n2 = int(keys["pk"]["n_squared"])
        rows = []
        for row in ciphers_batch:
            if len(row) != self._chunk_num:
                raise RuntimeError("decode_hamming_client: each inner list must have length == chunk_num")
            rows.append(_ciphertexts(row, n2))
        return self._ctx().decode_hamming(rows, self._chunk_num, self._chunk_len)

    # -- keys and configuration -------------------------------------------
    def get_pk_hex(self) -> tuple[str, str]:
        pk = self._need_keys("get_pk_hex")["pk"]
        return format(pk["n"], "x"), format(pk["n_squared"], "x")

    def get_keys_hex(self) -> tuple[str, str, str, str]:
        keys = self._need_keys("get_keys_hex")
        n, phi = keys["pk"]["n"], keys["sk"]["phi"]
        return format(n, "x"), format(keys["pk"]["n_squared"], "x"), format(phi, "x"), format(pow(phi, -1, n), "x")

    def stringify_pk(self) -> str:
        pk = self._need_keys("stringify_pk")["pk"]
        g_n = pk.get("g_n") or device_for(int(pk["n"])).modexp([int(pk["g"])], int(pk["n"]))[0]
        return json.dumps({"g": int(pk["g"]), "n": int(pk["n"]), "n_squared": int(pk["n_squared"]), "g_n": int(g_n)})

    def stringify_sk(self) -> str:
        sk = self._need_keys("stringify_sk")["sk"]
        return json.dumps({"phi": int(sk["phi"]), "a": int(sk["a"]), "g_a_inv": int(sk["g_a_inv"])})

    def stringify_config(self) -> str:
        return json.dumps({"message_chunks": int(self.message_chunks), "alpha_len": self.alpha_len,
                           "embed_len": self._embed_len, "key_len": self._key_len})

    def load_stringified_keys(self, pk: str, sk: str) -> None:
        p, s = json.loads(pk), json.loads(sk)
        n = int(p["n"])
        phi = int(s["phi"])
        if math.gcd(phi, n) != 1:
            raise RuntimeError("load_stringified_keys: phi^{-1} mod n does not exist")
        n2 = int(p["n_squared"])
        if n2.bit_length() > 4 * KEY_BITS:
            raise RuntimeError("load_stringified_keys: n_squared exceeds the supported width")
        a = int(s["a"])
        self.keys = {
            "pk": {"g": int(p["g"]), "n": n, "n_squared": n2, "g_n": int(p.get("g_n", 0)) or None},
            "sk": {"phi": phi, "a": a, "g_a_inv": int(s["g_a_inv"])},
            "g_table": {}, "noise_table": [], "key_len": 0, "message_chunks": 0,
        }
        if self.keys["pk"]["g_n"] is None:
            del self.keys["pk"]["g_n"]
        self.alpha_len = a.bit_length()
        self.message_chunks = 0

    def load_config(self, config: dict, tables: dict | None = None) -> None:
        if self.keys is None:
            raise RuntimeError("load_config: keys must be loaded first")
        keys = self.keys
        key_len = int(config["key_len"])
        if key_len > KEY_BITS:
            raise RuntimeError(f"load_config: key_len={key_len} exceeds KEY_BITS={KEY_BITS}")
        self._embed_len = int(config["embed_len"])
        self._key_len = key_len
        self.alpha_len = int(config["alpha_len"])
        self._chunk_len, self._chunk_num = chunk_layout(self._embed_len, self._key_len)
        self.message_chunks = int(config["message_chunks"])
        keys["message_chunks"] = self.message_chunks
        keys["key_len"] = key_len
        if tables is not None:
            if not isinstance(tables, dict):
                raise RuntimeError("load_config: tables must be a dict")
            g_table = _g_table_from_py(tables.get("g_table"), self.message_chunks)
            noise = [_as_int(v) for v in (tables.get("noise_table") or [])]
            if noise and len(noise) != 256:
                raise RuntimeError("load_config: noise_table size mismatch")
            keys["g_table"], keys["noise_table"] = g_table, noise
            if g_table and noise:
                self._install_tables()
        else:
            keys["g_table"], keys["noise_table"] = {}, []

    def dump_tables(self) -> dict:
        self._ensure_tables()
        return PaillierLookup.dump_tables(self._need_keys("dump_tables"))

    def dump_tables_bytes(self) -> dict:
        return self.dump_tables()

    def load_config_bytes(self, config: dict, tables: dict | None = None) -> None:
        self.load_config(config, tables)


class PaillierGPUClient:
    """Textbook-Paillier Hamming client on the B200 (hex-string ciphertexts)."""

    @staticmethod
    def max_key_len() -> int:
        return KEY_BITS

    def __init__(self, embed_len: int = 512, key_len: int = 1024, skip_key_gen: bool = False) -> None:
        if key_len > KEY_BITS:
            raise RuntimeError(f"PaillierGPUClient: key_len={key_len} exceeds KEY_BITS={KEY_BITS}")
        self._embed_len = int(embed_len)
        self._key_len = int(key_len)
        self._chunk_len, self._chunk_num = chunk_layout(self._embed_len, self._key_len)
        self.keys = None if skip_key_gen else Paillier.key_gen(self._key_len)
        device_for_probe()

    embed_len = property(lambda self: self._embed_len)
    key_len = property(lambda self: self._key_len)
    chunk_len = property(lambda self: self._chunk_len)
    chunk_num = property(lambda self: self._chunk_num)

    def _need_keys(self, what: str) -> dict:
        if self.keys is None:
            raise RuntimeError(f"{what}: keys not initialized")
        return self.keys

    def encrypt(self, embeddings: Sequence[Sequence[int]]) -> list[list[str]]:
        """paillier_GPU_client.cu:873-974: each embedding's bits padded to "0b"
        pairs, cut into chunk_len-bit chunks read most significant first (the
        reference CPU client's int(bits, 2)), encrypted with r drawn as in
        Paillier.encrypt; ciphertexts as hex strings formatted on the device."""
        keys = self._need_keys("encrypt")
        if len(embeddings) == 0:
            return []
        bits = _bits_array(embeddings, self._embed_len)
        ctx = device_for(int(keys["pk"]["n"]))
        m = _chunk_plaintexts(bits, self._chunk_len, self._chunk_num, ctx.words)
        plaintexts = [int.from_bytes(row.tobytes(), "little") for row in m]
        cts = Paillier.encrypt_batch(plaintexts, keys["pk"])
        hexes = ctx.to_hex(ctx.limbs(cts))
        return [hexes[i * self._chunk_num:(i + 1) * self._chunk_num] for i in range(len(bits))]

    def encode_hamming_client(self, ct1: Sequence[str], ct2: Sequence[str]) -> list[str]:
        keys = self._need_keys("encode_hamming_client")
        return PaillierGPUClient.encode_hamming_server(ct1, ct2, {"n_squared": format(keys["pk"]["n_squared"], "x")})

    @staticmethod
    def encode_hamming_server(ct1: Sequence[str], ct2: Sequence[str], pk: dict) -> list[str]:
        """ct1[i] * ct2[i] mod n^2 on hex strings (paillier_GPU_client.cu:672-732):
        parsing, the products and formatting all on the device."""
        if len(ct1) != len(ct2):
            raise RuntimeError("encode_hamming_*: ct1 and ct2 must have the same length")
        n2 = int(str(pk["n_squared"]), 16)
        n = math.isqrt(n2)
        if n * n != n2:
            raise RuntimeError("encode_hamming_server: n_squared is not a perfect square")
        if not ct1:
            return []
        ctx = device_for(n)
        try:
            a = ctx.from_hex([str(c) for c in ct1])
            b = ctx.from_hex([str(c) for c in ct2])
        except ValueError as exc:
            raise RuntimeError(str(exc)) from exc
        out = ctx.empty(len(ct1))
        ctx.mulmod_array(a, b, out, len(ct1))
        return ctx.to_hex(out)

    def decode_hamming_client(self, ciphers_hex_batch: Sequence[Sequence[str]]) -> list[int]:
        """paillier_GPU_client.cu:995-1038 on the device: hex parsing, c^phi,
        L(), * phi^-1 and the odd-bit count."""
        keys = self._need_keys("decode_hamming_client")
        flat = []
        for row in ciphers_hex_batch:
            if len(row) != self._chunk_num:
                raise RuntimeError("decode_hamming_client: each inner list must have length == chunk_num")
            flat.extend(str(c) for c in row)
        if not flat:
            return []
        ctx = device_for(int(keys["pk"]["n"]), (int(keys["sk"]["phi"]), int(keys["sk"]["inv"])),
                         phi=keys["sk"]["phi"])
        try:
            c = ctx.from_hex(flat)
        except ValueError as exc:
            raise RuntimeError(str(exc)) from exc
        vectors = len(flat) // self._chunk_num
        out = np.zeros(vectors, dtype=np.int64)
        ctx.decode_array(c, vectors, self._chunk_num, self._chunk_len, out)
        return [int(v) for v in out]

    def get_pk_hex(self) -> tuple[str, str]:
        pk = self._need_keys("get_pk_hex")["pk"]
        return format(pk["n"], "x"), format(pk["n_squared"], "x")

    def get_keys_hex(self) -> tuple[str, str, str, str]:
        keys = self._need_keys("get_keys_hex")
        return (format(keys["pk"]["n"], "x"), format(keys["pk"]["n_squared"], "x"),
                format(keys["sk"]["phi"], "x"), format(keys["sk"]["inv"], "x"))

    def stringify_pk(self) -> str:
        pk = self._need_keys("stringify_pk")["pk"]
        return json.dumps({"g": str(pk["n"] + 1), "n": str(pk["n"]), "n_squared": str(pk["n_squared"])})

    def stringify_sk(self) -> str:
        sk = self._need_keys("stringify_sk")["sk"]
        return json.dumps({"phi": str(sk["phi"]), "inv": str(sk["inv"])})

    def stringify_config(self) -> str:
        return json.dumps({"embed_len": self._embed_len, "key_len": self._key_len})

    def load_stringified_keys(self, pk: str, sk: str) -> None:
        p, s = json.loads(pk), json.loads(sk)
        n = int(str(p["n"]))
        n2 = int(str(p["n_squared"]))
        if n2.bit_length() > 4 * KEY_BITS:
            raise RuntimeError("load_stringified_keys: n_squared exceeds the supported width")
        self.keys = {"pk": {"g": n + 1, "n": n, "n_squared": n2},
                     "sk": {"phi": int(str(s["phi"])), "inv": int(str(s["inv"]))}}

    def load_config(self, config: dict) -> None:
        key_len = int(config["key_len"])
        if key_len > KEY_BITS:
            raise RuntimeError(f"load_config: key_len={key_len} exceeds KEY_BITS={KEY_BITS}")
        self._embed_len = int(config["embed_len"])
        self._key_len = key_len
        self._chunk_len, self._chunk_num = chunk_layout(self._embed_len, self._key_len)


def device_for_probe() -> None:
    """Fail at construction when the library or a CUDA device is missing."""
    from cuhepy_b200 import _native

    _native.paillier_lib()
    from cuhepy_b200.paillier.gpu import PaillierDevice

    PaillierDevice(3).close()
