"""Generates the golden fixtures in tests/golden/ (run where the reference tree and python-xxhash are
available):

    GS_REFERENCE_TREE=<reference checkout> python tests/golden/make_golden.py

GS_REFERENCE_TREE defaults to a directory named `reference` beside this repository's root.

* xxh3_vectors.json   XXH3_64bits_withSeed of 8-byte keys from python-xxhash (libxxhash), the hash
                      the reference binds in include/types.h:8-9.
* geometry.json       num_buckets per (V, sketches_factor) read from the reference's own CCSketchAlg
                      (get_desired_updates_per_batch = num_buckets*16/4, include/cc_sketch_alg.h:147-151),
                      compiled into oracle/_ref/libgsref.so.
* multiples_1024_stream.npy
                      an 8528-record insert/delete stream whose final graph is the reference's
                      test/res/multiples_graph_1024.txt fixture (edges {i, j}: 2 <= i, j a multiple of i,
                      j < 1024; 78 connected components, test/cc_alg_test.cpp:41-57).  The edge set is
                      rebuilt from that rule and checked against the reference file here; the record
                      order and the delete/reinsert churn (6867 inserts, 1661 deletes, as in
                      multiples_graph_1024_stream.data) are our own seeded choice.
* multiples_graph_1024_stream.data
                      the reference's own binary stream fixture (test/res/multiples_graph_1024_stream.data,
                      replayed by test/cc_alg_test.cpp:300-350), copied byte for byte: {u32 V, u64 n}
                      then n packed {u8 type, u32 src, u32 dst} records.
* ref_digests.json    sha256 of the reference CCSketchAlg's write_binary sketch bytes, its component
                      count and Boruvka rounds, for seeded streams (the plain-CC ER stream among them)
                      and for the records of the reference's binary fixture in file order.
"""
from __future__ import annotations

import hashlib
import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
from stream_file import read_stream_file  # noqa: E402

REF_TREE = os.environ.get("GS_REFERENCE_TREE", os.path.join(os.path.dirname(ROOT), "reference"))
FIXTURE = "multiples_graph_1024_stream.data"


def copy_reference_fixture() -> None:
    with open(os.path.join(REF_TREE, "test", "res", FIXTURE), "rb") as f:
        data = f.read()
    with open(os.path.join(HERE, FIXTURE), "wb") as f:
        f.write(data)


def multiples_edges(V: int = 1024) -> np.ndarray:
    out = [(i, j) for i in range(2, V) for j in range(2 * i, V, i)]
    return np.asarray(out, np.uint32)


def multiples_stream(seed: int = 0x5EED0078) -> np.ndarray:
    """Final graph = multiples graph; 1661 extra edges are inserted and later deleted."""
    rng = np.random.default_rng(seed)
    edges = multiples_edges()
    present = set(map(tuple, edges.tolist()))
    extra = []
    while len(extra) < 1661:
        a, b = sorted(rng.integers(0, 1024, 2).tolist())
        if a != b and (a, b) not in present and (a, b) not in extra:
            extra.append((a, b))
    extra = np.asarray(extra, np.uint32)
    ins = np.concatenate([edges, extra])
    ins = ins[rng.permutation(len(ins))]
    # each extra edge is deleted at a random point after its insert
    pos = {tuple(e): k for k, e in enumerate(ins.tolist())}
    recs = [(k, 0, tuple(e)) for k, e in enumerate(ins.tolist())]
    for e in extra.tolist():
        k = pos[tuple(e)]
        recs.append((rng.uniform(k + 0.5, len(ins)), 1, tuple(e)))
    recs.sort(key=lambda r: r[0])
    arr = np.asarray([r[2] for r in recs], np.uint32)
    flip = rng.random(len(arr)) < 0.5  # record orientation does not matter; exercise both
    arr[flip] = arr[flip][:, ::-1]
    return arr


def check_against_reference_fixture(edges: np.ndarray) -> None:
    path = os.path.join(REF_TREE, "test", "res", "multiples_graph_1024.txt")
    with open(path) as f:
        lines = f.read().split("\n")
    V, E = map(int, lines[0].split())
    ref = {tuple(sorted(map(int, l.split()))) for l in lines[1:] if l.strip()}
    assert V == 1024 and E == len(ref) == len(edges), (V, E, len(ref), len(edges))
    assert ref == set(map(tuple, edges.tolist())), "multiples graph rule differs from the reference fixture"
    # the binary twin: same final graph, 8528 records of which 1661 deletes
    with open(os.path.join(REF_TREE, "test", "res", "multiples_graph_1024_stream.data"), "rb") as f:
        d = f.read()
    v, n = struct.unpack_from("<IQ", d, 0)
    types = [d[12 + 9 * k] for k in range(n)]
    assert (v, n, types.count(1)) == (1024, 8528, 1661), (v, n, types.count(1))


def xxh3_vectors() -> list:
    import xxhash
    rng = np.random.default_rng(0x78683)
    keys = [0, 1, 2**32 - 1, 2**32, 2**63, 2**64 - 1, 0x00000001_00000002]
    seeds = [0, 1, 5, 0xC0FFEE, 2**31, 2**32 - 1, 2**32, 2**63, 2**64 - 1, 0xDEADBEEF_CAFEBABE]
    keys += [int(x) for x in rng.integers(0, 2**63, 40, dtype=np.int64)]
    seeds += [int(x) for x in rng.integers(0, 2**63, 20, dtype=np.int64)]
    out = []
    for k in keys:
        for s in seeds[:6] if k > 2**40 else seeds:
            out.append([str(k), str(s), str(xxhash.xxh3_64_intdigest(struct.pack("<Q", k), s))])
    # column seeds seed+5c of one sketch, the way Bucket_Boruvka hashes them
    for c in range(24):
        k = (17 << 32) | 4242
        s = 0xC0FFEE + 5 * c
        out.append([str(k), str(s), str(xxhash.xxh3_64_intdigest(struct.pack("<Q", k), s))])
    return out


def geometry_table() -> list:
    from oracle import RefCC
    rows = []
    for V in [2, 3, 17, 256, 1000, 1024, 4096, 16384, 65536, 131072, 1 << 20]:
        for f in [1.0, 1.5, 3.0]:
            if V > 4096 and f != 1.0 and V != 131072:
                continue
            if V >= 1 << 17 and f == 3.0:
                continue
            r = RefCC(V, 1, f)
            nb = int(r.L.gsref_cc_desired_batch(r.h)) // 4
            r.close()
            rows.append([V, f, nb])
    return rows


def ref_digests() -> list:
    import gpusketch_b200 as gs
    from oracle import RefCC
    cases = [
        # name, V, sketch seed, stream
        ("plain_cc_er1024", 1024, 0xC0FFEE, lambda: gs.er_stream(1024, 0.05, 0x5EED0001, 0.10, 0.5)),
        ("multiples_1024", 1024, 0xC0FFEE, lambda: np.load(os.path.join(HERE, "multiples_1024_stream.npy"))),
        ("er256_sparse", 256, 7, lambda: gs.er_stream(256, 0.01, 11, 0.5, 0.2)),
        ("er4096", 4096, 0x1234_5678_9ABC_DEF0, lambda: gs.er_stream(4096, 0.002, 13, 0.1, 0.5)),
        ("rmat_v2p12", 4096, 2**63 + 5, lambda: gs.rmat_stream(12, 40000, 0x5EED0002)),
        ("multiples_file_1024", 1024, 0xC0FFEE, lambda: read_stream_file(os.path.join(HERE, FIXTURE))[2]),
    ]
    out = []
    for name, V, seed, mk in cases:
        pairs = mk()
        r = RefCC(V, seed, 1.0)
        for a, b in pairs.tolist():
            r.update(a, b, 0)
        sk = r.sketch_bytes()
        labels, ncc, rounds = r.connected_components()
        r.close()
        out.append(dict(name=name, V=V, seed=str(seed), records=int(len(pairs)),
                        pairs_sha256=hashlib.sha256(np.ascontiguousarray(pairs, np.uint32).tobytes()).hexdigest(),
                        sketch_sha256=hashlib.sha256(sk).hexdigest(), num_cc=int(ncc), rounds=int(rounds)))
    return out


def main() -> None:
    edges = multiples_edges()
    if os.path.isdir(REF_TREE):
        check_against_reference_fixture(edges)
        copy_reference_fixture()
    np.save(os.path.join(HERE, "multiples_1024_stream.npy"), multiples_stream())
    with open(os.path.join(HERE, "xxh3_vectors.json"), "w") as f:
        json.dump(xxh3_vectors(), f, indent=0)
    with open(os.path.join(HERE, "geometry.json"), "w") as f:
        json.dump(geometry_table(), f)
    with open(os.path.join(HERE, "ref_digests.json"), "w") as f:
        json.dump(ref_digests(), f, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
