"""Writes hash_vectors.json: the reference's own hash functions evaluated on a fixed
key set. The values come from src/dpu/src/hash.c of yonsei-hpcp/spid-join, compiled
from source by `make -C oracle ref` into oracle/_ref/libref_hash.so (needs the
reference tree; the JSON is committed so the tests need neither)."""
import ctypes
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "..", "oracle", "_ref", "libref_hash.so")


def keys():
    ks = list(range(0, 300))
    ks += [1 << b for b in range(32)] + [(1 << b) - 1 for b in range(1, 33)]
    x = 0x5EED5EED
    for _ in range(700):  # xorshift32 stream, fixed
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        ks.append(x)
    return ks


def main():
    L = ctypes.CDLL(REF)
    names = ["glb_partition_hash", "local_partition_hash", "join_hash", "join_hash2"]
    for n in names:
        getattr(L, n).restype = ctypes.c_uint32
        getattr(L, n).argtypes = [ctypes.c_uint32]
    crc = (ctypes.c_uint32 * 256).in_dll(L, "crctab")
    out = {"source": "src/dpu/src/hash.c (reference, compiled with -DCRC)",
           "crctab": [int(crc[i]) for i in range(256)],
           "keys": keys()}
    for n in names:
        out[n] = [int(getattr(L, n)(k)) for k in out["keys"]]
    with open(os.path.join(HERE, "hash_vectors.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
