"""The reference-named Paillier client APIs, driven on the device.

The north star's drop-in surface is the client layer: the Hamming clients
``PaillierLookupClient`` / ``PaillierClient`` (src/cuhepy/hamming/
paillier_lookup.py:245-425, hamming/paillier.py:113-231) and the classes they
load, ``PaillierGPULookupClient`` / ``PaillierGPUClient`` (method sets of
paillier_GPU_lookup_client.cu:2673-2722 and paillier_GPU_client.cu:1136-1166).
These tests drive that layer with the golden keys made by the reference code
and the reference's recorded random draws replayed through ``secrets``, so
every ciphertext must equal the reference's byte for byte; they follow the
flow of the reference's own GPU client tests (test_GPU_paillier_clients.py:
58-141: encrypt -> encode -> decode, key reload, pickling, CPU<->GPU
interop), with the oracle standing in for the reference's CPU backend.
Integer work: equality is exact.
"""

import json
import pickle
import random

import pytest

from conftest import hx, load_golden
from oracle import paillier as oracle

pytestmark = pytest.mark.gpu


class Replay:
    """A ``secrets`` stand-in returning recorded draws in order."""

    def __init__(self, values):
        self.values = list(values)

    def randbelow(self, bound):
        value = self.values.pop(0)
        assert 0 <= value < bound
        return value

    def randbits(self, k):
        raise AssertionError("no bit draws expected")


def _hamming(a, b):
    return sum(int(x != y) for x, y in zip(a, b))


def _lookup_golden():
    data = load_golden("lookup_1024.json")
    pk = {k: hx(v) for k, v in data["pk"].items()}
    sk = {k: hx(v) for k, v in data["sk"].items()}
    return data, pk, sk


def _lookup_client(data, pk, sk, monkeypatch):
    """A client with the golden keys; its tables are built on first use with
    the reference's 256 noise exponents replayed."""
    from cuhepy_b200.hamming.paillier_lookup import PaillierLookupClient
    from cuhepy_b200.paillier import lookup

    client = PaillierLookupClient(embed_len=512, key_len=1024, skip_key_gen=True, device="gpu")
    assert client.device == "gpu"
    client.load_stringified_keys(json.dumps(pk), json.dumps(sk))
    client.load_config({"message_chunks": data["message_chunks"], "alpha_len": data["alpha_len"],
                        "embed_len": 512, "key_len": 1024})
    monkeypatch.setattr(lookup, "secrets", Replay([hx(r) - 1 for r in data["noise_exponents"]]))
    tables = client.dump_tables()
    width = (pk["n_squared"].bit_length() + 7) // 8
    rows = [tables["g_table"][i] for i in range(data["message_chunks"])]
    assert oracle.table_digest(rows, width) == data["g_table_sha256"]
    assert oracle.table_digest(tables["noise_table"], width) == data["noise_table_sha256"]
    return client


def test_lookup_client_reproduces_reference_hamming_flow(monkeypatch):
    """encrypt_vec_one / encrypt_vec_batch / encode_hamming_server /
    decode_hamming_client_one / _batch against the reference client's
    recorded ciphertexts and distances."""
    from cuhepy_b200.paillier import clients

    data, pk, sk = _lookup_golden()
    client = _lookup_client(data, pk, sk, monkeypatch)
    vectors = data["hamming"]["vectors"]
    bits = [[int(b) for b in v["bits"]] for v in vectors]
    monkeypatch.setattr(clients, "secrets", Replay(vectors[0]["indices"]))
    one = client.encrypt_vec_one(bits[0])
    assert one == [hx(c) for c in vectors[0]["c"]]
    monkeypatch.setattr(clients, "secrets", Replay([i for v in vectors for i in v["indices"]]))
    batch = client.encrypt_vec_batch(bits)
    assert batch == [[hx(c) for c in v["c"]] for v in vectors]
    encoded = []
    for pair in data["hamming"]["pairs"]:
        server = client.encode_hamming_server(batch[pair["i"]], batch[pair["j"]])
        assert server == [hx(pair["c"])]
        assert client.decode_hamming_client_one(server) == pair["distance"]
        assert pair["distance"] == _hamming(bits[pair["i"]], bits[pair["j"]])
        encoded.append(server)
    assert client.decode_hamming_client_batch(encoded) == [p["distance"] for p in data["hamming"]["pairs"]]
    # ciphertexts given as little-endian bytes, as the reference accepts
    as_bytes = [c.to_bytes(512, "little") for c in encoded[0]]
    assert client.decode_hamming_client_one(as_bytes) == data["hamming"]["pairs"][0]["distance"]


def test_lookup_client_key_reload_and_pickle(monkeypatch):
    """stringify_pk/_sk/_config -> a fresh client -> load_stringified_keys +
    load_config(precomputed_tables=dump_tables()) gives the same ciphertexts;
    so does a pickle round trip (paillier_lookup.py:402-425)."""
    from cuhepy_b200.hamming.paillier_lookup import PaillierLookupClient
    from cuhepy_b200.paillier import clients

    data, pk, sk = _lookup_golden()
    client = _lookup_client(data, pk, sk, monkeypatch)
    assert json.loads(client.stringify_pk()) == pk
    assert json.loads(client.stringify_sk()) == sk
    config = json.loads(client.stringify_config())
    assert config == {"message_chunks": 256, "alpha_len": 280, "embed_len": 512, "key_len": 1024}
    clone = PaillierLookupClient(embed_len=512, key_len=1024, alpha_len=config["alpha_len"], skip_key_gen=True,
                                 device="gpu")
    clone.load_stringified_keys(client.stringify_pk(), client.stringify_sk())
    clone.load_config(config, precomputed_tables=client.dump_tables())
    restored = pickle.loads(pickle.dumps(client))
    vector = data["hamming"]["vectors"][2]
    bits = [int(b) for b in vector["bits"]]
    for other in (clone, restored):
        assert json.loads(other.stringify_pk()) == pk and json.loads(other.stringify_sk()) == sk
        assert json.loads(other.stringify_config()) == config
        monkeypatch.setattr(clients, "secrets", Replay(vector["indices"]))
        assert other.encrypt_vec_one(bits) == [hx(c) for c in vector["c"]]
        pair = data["hamming"]["pairs"][0]
        assert other.decode_hamming_client_one([hx(pair["c"])]) == pair["distance"]


def test_lookup_client_interop_with_cpu_oracle(monkeypatch):
    """Keys are portable between the device and the CPU restatement of the
    reference: CPU ciphertexts decode on the device and device ciphertexts
    decrypt on the CPU (test_GPU_paillier_clients.py:98-128)."""
    data, pk, sk = _lookup_golden()
    client = _lookup_client(data, pk, sk, monkeypatch)
    keys = {"pk": pk, "sk": sk}
    tables = client.dump_tables()
    table = [tables["g_table"][i] for i in range(data["message_chunks"])]
    noise = tables["noise_table"]
    rng = random.Random(98)
    a = [rng.getrandbits(1) for _ in range(512)]
    b = [rng.getrandbits(1) for _ in range(512)]
    expected = _hamming(a, b)
    (ma,) = oracle.encode_bits(a, 1024)
    (mb,) = oracle.encode_bits(b, 1024)
    cpu_a = oracle.lookup_encrypt(ma, pk, table, noise, [rng.randrange(256) for _ in range(14)], 256)
    cpu_b = oracle.lookup_encrypt(mb, pk, table, noise, [rng.randrange(256) for _ in range(14)], 256)
    # evaluate and decode on the device
    assert client.decode_hamming_client_one(client.encode_hamming_server([cpu_a], [cpu_b])) == expected
    # encrypt on the device, evaluate and decrypt on the CPU
    dev_a, dev_b = client.encrypt_vec_one(a), client.encrypt_vec_one(b)
    server = oracle.add(dev_a[0], dev_b[0], pk["n_squared"])
    assert oracle.decode_distance([oracle.lookup_decrypt(server, keys)], 1024) == expected
    assert client.encode_hamming_server(dev_a, dev_b) == [server]


def test_lookup_gpu_class_method_set(monkeypatch):
    """PaillierGPULookupClient's own methods: encrypt_cts / decrypt_cts with
    the reference's recorded noise indices, encode_hamming_client, hex key
    accessors, load_config with tables, and the reference's error messages."""
    from cuhepy_b200.paillier import clients
    from cuhepy_b200.paillier.clients import PaillierGPULookupClient

    data, pk, sk = _lookup_golden()
    wrapper = _lookup_client(data, pk, sk, monkeypatch)
    tables = wrapper.dump_tables()
    gpu = PaillierGPULookupClient(embed_len=512, key_len=1024, skip_key_gen=True)
    with pytest.raises(RuntimeError, match="^load_config: keys must be loaded first$"):
        gpu.load_config({"message_chunks": 256, "alpha_len": 280, "embed_len": 512, "key_len": 1024})
    with pytest.raises(RuntimeError, match="^encrypt: keys not initialized$"):
        gpu.encrypt([[0] * 512])
    with pytest.raises(RuntimeError, match="^decode_hamming_client: keys not initialized$"):
        gpu.decode_hamming_client([[1]])
    gpu.load_stringified_keys(json.dumps(pk), json.dumps(sk))
    gpu.load_config({"message_chunks": 256, "alpha_len": 280, "embed_len": 512, "key_len": 1024}, tables)
    assert (gpu.embed_len, gpu.key_len, gpu.chunk_len, gpu.chunk_num) == (512, 1024, 2048, 1)
    assert PaillierGPULookupClient.max_key_len() == clients.KEY_BITS
    n, n2 = gpu.get_pk_hex()
    assert (int(n, 16), int(n2, 16)) == (pk["n"], pk["n_squared"])
    cases = data["encrypt"]
    monkeypatch.setattr(clients, "secrets", Replay([i for c in cases for i in c["indices"]]))
    cts = gpu.encrypt_cts([hx(c["m"]) for c in cases])
    assert cts == [hx(c["c"]) for c in cases]
    assert gpu.decrypt_cts(cts) == [hx(c["d"]) for c in cases]
    sums = gpu.encode_hamming_client([cts[s["i"]] for s in data["add"]], [cts[s["j"]] for s in data["add"]])
    assert sums == [hx(s["c"]) for s in data["add"]]
    assert gpu.decrypt_cts(sums) == [hx(s["m"]) for s in data["add"]]
    # values given as decimal / hex strings or LE bytes convert like ints
    assert gpu.decrypt_cts([str(cts[0]), hex(cts[1]), cts[2].to_bytes(512, "little")]) == \
        [hx(c["d"]) for c in cases[:3]]
    static = PaillierGPULookupClient.encode_hamming_server([cts[0]], [cts[1]], {"n_squared": pk["n_squared"]})
    assert static == [cts[0] * cts[1] % pk["n_squared"]]
    with pytest.raises(RuntimeError, match="^encode_hamming_server: pk must contain n_squared$"):
        PaillierGPULookupClient.encode_hamming_server([cts[0]], [cts[1]], {"n": pk["n"]})
    with pytest.raises(RuntimeError, match="^encode_hamming_server: ct1 and ct2 must have the same length$"):
        PaillierGPULookupClient.encode_hamming_server([cts[0]], [], pk)
    with pytest.raises(RuntimeError, match=r"^encrypt_cts: plaintext out of range \[0, n\)$"):
        gpu.encrypt_cts([pk["n"]])
    with pytest.raises(RuntimeError, match="^encrypt: each embedding must have length == embed_len$"):
        gpu.encrypt([[0] * 511])
    with pytest.raises(RuntimeError, match="^encrypt: embeddings must be binary 0/1$"):
        gpu.encrypt([[0] * 511 + [2]])
    with pytest.raises(RuntimeError, match="^decode_hamming_client: each inner list must have length == chunk_num$"):
        gpu.decode_hamming_client([[cts[0], cts[1]]])
    # table parsing follows g_table_from_py (paillier_GPU_lookup_client.cu:1377-1426): rows by int or
    # str key, or a sequence of exactly message_chunks rows of 256 entries
    config = {"message_chunks": 256, "alpha_len": 280, "embed_len": 512, "key_len": 1024}
    by_str = {"g_table": {str(k): v for k, v in tables["g_table"].items()}, "noise_table": tables["noise_table"]}
    gpu.load_config(config, by_str)
    monkeypatch.setattr(clients, "secrets", Replay(cases[0]["indices"]))
    assert gpu.encrypt_cts([hx(cases[0]["m"])]) == [hx(cases[0]["c"])]
    rows = [tables["g_table"][i] for i in range(256)]
    with pytest.raises(RuntimeError, match="^g_table missing row$"):
        gpu.load_config(dict(config, message_chunks=257), tables)
    with pytest.raises(RuntimeError, match="^g_table outer length mismatch$"):
        gpu.load_config(config, {"g_table": rows[:255], "noise_table": tables["noise_table"]})
    with pytest.raises(RuntimeError, match="^g_table row length mismatch$"):
        gpu.load_config(config, {"g_table": [r[:255] for r in rows], "noise_table": tables["noise_table"]})
    with pytest.raises(RuntimeError, match="^load_config: noise_table size mismatch$"):
        gpu.load_config(config, {"g_table": rows, "noise_table": tables["noise_table"][:255]})
    with pytest.raises(RuntimeError, match="^load_config: tables must be a dict$"):
        gpu.load_config(config, [rows])


def test_plain_client_hex_api(monkeypatch):
    """PaillierGPUClient's hex-string API and the PaillierClient wrapper with
    the reference's golden keys; r replayed through scheme.secrets."""
    from cuhepy_b200.hamming.paillier import PaillierClient
    from cuhepy_b200.paillier import scheme
    from cuhepy_b200.paillier.clients import PaillierGPUClient

    data = load_golden("paillier_1024.json")
    pk = {k: hx(v) for k, v in data["pk"].items()}
    sk = {k: hx(v) for k, v in data["sk"].items()}
    keys = {"pk": pk, "sk": sk}
    client = PaillierClient(embed_len=512, key_len=1024, skip_key_gen=True, device="gpu")
    pk_json = json.dumps({"g": str(pk["g"]), "n": str(pk["n"]), "n_squared": str(pk["n_squared"])})
    sk_json = json.dumps({"phi": str(sk["phi"]), "inv": str(sk["inv"])})
    client.load_stringified_keys(pk_json, sk_json)
    client.load_config({"embed_len": 512, "key_len": 1024, "device": "gpu"})
    assert json.loads(client.stringify_pk()) == json.loads(pk_json)
    assert json.loads(client.stringify_sk()) == json.loads(sk_json)
    assert json.loads(client.stringify_config()) == {"embed_len": 512, "key_len": 1024}
    rng = random.Random(5)
    vecs = [[rng.getrandbits(1) for _ in range(512)] for _ in range(3)]
    rs = [rng.randrange(1, pk["n"]) for _ in range(3)]
    monkeypatch.setattr(scheme, "secrets", Replay([r - 1 for r in rs]))
    cts = client.encrypt_vec_batch(vecs)
    want = [[oracle.encrypt(oracle.encode_bits(v, 1024)[0], r, pk)] for v, r in zip(vecs, rs)]
    assert cts == want
    server = client.encode_hamming_server(cts[0], cts[1])
    assert server == [cts[0][0] * cts[1][0] % pk["n_squared"]]
    assert client.decode_hamming_client_one(server) == _hamming(vecs[0], vecs[1])
    server2 = client.encode_hamming_server(cts[1], cts[2])
    assert client.decode_hamming_client_batch([server, server2]) == [_hamming(vecs[0], vecs[1]),
                                                                     _hamming(vecs[1], vecs[2])]
    # the hex-string class itself, with the golden ciphertext pairs
    gpu = client.client
    assert isinstance(gpu, PaillierGPUClient)
    cs = [format(hx(c["c"]), "x") for c in data["encrypt"]]
    pairs = data["add"]
    out = PaillierGPUClient.encode_hamming_server([cs[p["i"]] for p in pairs], [cs[p["j"]] for p in pairs],
                                                  {"n_squared": format(pk["n_squared"], "x")})
    assert out == [format(hx(p["c"]), "x") for p in pairs]
    assert gpu.encode_hamming_client(["0x" + cs[0].upper()], [cs[1]]) == [format(hx(pairs[0]["c"]), "x")]
    assert gpu.get_keys_hex() == tuple(format(v, "x") for v in (pk["n"], pk["n_squared"], sk["phi"], sk["inv"]))
    # a device ciphertext decrypts on the CPU and a CPU ciphertext decodes on the device
    assert oracle.decode_distance([oracle.decrypt(server[0], keys)], 1024) == _hamming(vecs[0], vecs[1])
    cpu = [oracle.add(want[1][0], want[2][0], pk["n_squared"])]
    assert gpu.decode_hamming_client([[format(cpu[0], "x")]]) == [_hamming(vecs[1], vecs[2])]
    with pytest.raises(RuntimeError, match="^encrypt: embeddings must be binary 0/1$"):
        gpu.encrypt([[0] * 511 + [3]])
    with pytest.raises(RuntimeError, match="^encode_hamming_\\*: ct1 and ct2 must have the same length$"):
        PaillierGPUClient.encode_hamming_server(cs[:2], cs[:1], {"n_squared": format(pk["n_squared"], "x")})
    with pytest.raises(ValueError, match="Embedding length 3 does not match expected 512"):
        client.encrypt_vec_one([0, 1, 0])


def test_reference_gpu_client_flow_small_embedding():
    """The reference's own GPU client test flow (embed_len 8, fresh keys):
    encrypt -> encode -> decode, then a key reload into a new client
    (test_GPU_paillier_clients.py:58-95), for both client kinds."""
    from cuhepy_b200.hamming.paillier import PaillierClient
    from cuhepy_b200.hamming.paillier_lookup import PaillierLookupClient

    vectors = [[0, 1, 0, 1, 1, 0, 1, 0], [1, 1, 0, 0, 1, 0, 0, 1], [1, 0, 1, 0, 1, 1, 0, 0]]
    for cls in (PaillierClient, PaillierLookupClient):
        assert cls.has_gpu()
        client = cls(embed_len=8, key_len=1024, device="gpu")
        one = client.encrypt_vec_one(vectors[0])
        batch = client.encrypt_vec_batch(vectors)
        assert len(batch) == 3 and len(one) == len(batch[0]) == 1
        assert client.decode_hamming_client_one(client.encode_hamming_server(one, batch[1])) == \
            _hamming(vectors[0], vectors[1])
        encoded = [client.encode_hamming_server(batch[0], batch[1]), client.encode_hamming_server(batch[1], batch[2])]
        assert client.decode_hamming_client_batch(encoded) == [_hamming(vectors[0], vectors[1]),
                                                                _hamming(vectors[1], vectors[2])]
        config = json.loads(client.stringify_config())
        kwargs = {"alpha_len": config["alpha_len"]} if cls is PaillierLookupClient else {}
        clone = cls(embed_len=8, key_len=1024, skip_key_gen=True, device="gpu", **kwargs)
        clone.load_stringified_keys(client.stringify_pk(), client.stringify_sk())
        if cls is PaillierLookupClient:
            clone.load_config(config, precomputed_tables=client.dump_tables())
        else:
            clone.load_config(config)
        again = clone.encode_hamming_server(clone.encrypt_vec_one(vectors[0]), clone.encrypt_vec_one(vectors[1]))
        assert clone.decode_hamming_client_one(again) == _hamming(vectors[0], vectors[1])
        assert json.loads(clone.stringify_config()) == config


def test_hex_wire_format_on_the_device():
    """Hex strings <-> limbs parsed and formatted on the device, with the
    reference's hex_to_le_words / le_words_to_hex semantics
    (paillier_GPU_client.cu:218-262): optional 0x / 0X prefix, either case,
    leading zeros, digits beyond the width dropped, "Invalid hex digit"
    otherwise; values at or above n^2 reduced when asked."""
    from cuhepy_b200.paillier.clients import PaillierGPUClient
    from cuhepy_b200.paillier.gpu import device_for

    data = load_golden("paillier_1024.json")
    n2 = hx(data["pk"]["n_squared"])
    n = hx(data["pk"]["n"])
    ctx = device_for(n)
    width = 32 * ctx.words
    rng = random.Random(16)
    vals = [0, 1, n2 - 1, n2, n2 + 5, (1 << width) - 1] + [rng.randrange(1 << width) for _ in range(300)]
    texts = [format(v, "x") for v in vals]
    texts[2] = "0x" + texts[2].upper()
    texts[3] = "000" + texts[3]
    texts.append("")                                  # the reference reads an empty string as 0
    texts.append("f" * 8 + format(12345, "x").zfill(8 * ctx.words))  # digits beyond the width are dropped
    vals += [0, 12345]
    from cuhepy_b200._limbs import from_limbs

    raw = from_limbs(ctx.from_hex(texts, reduce=False))
    assert raw == vals
    reduced = from_limbs(ctx.from_hex(texts))
    assert reduced == [v % n2 for v in vals]
    assert ctx.to_hex(ctx.limbs(reduced)) == [format(v, "x") for v in reduced]
    with pytest.raises(ValueError, match="Invalid hex digit"):
        ctx.from_hex(["12g4"])
    with pytest.raises(ValueError, match="Invalid hex digit"):
        ctx.from_hex(["ab cd"])
    with pytest.raises(ValueError, match="Invalid hex digit"):
        ctx.from_hex(["é"])
    # the client's products reduce inputs of any width, as the reference's CGBN kernel does
    a, b = vals[10], vals[11]
    out = PaillierGPUClient.encode_hamming_server([format(a, "x")], [format(b, "x")], {"n_squared": format(n2, "x")})
    assert out == [format(a * b % n2, "x")]
    with pytest.raises(RuntimeError, match="Invalid hex digit"):
        PaillierGPUClient.encode_hamming_server(["zz"], ["1"], {"n_squared": format(n2, "x")})
