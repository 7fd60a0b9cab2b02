"""Reader / writer of the binary graph-stream format of the reference's tools and tests
(test/res/multiples_graph_1024_stream.data): a header {u32 num_vertices, u64 num_updates} and then
num_updates packed 9-byte records {u8 type (0 insert, 1 delete), u32 src, u32 dst}."""
import os
import struct

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REFERENCE_FIXTURE = os.path.join(GOLDEN, "multiples_graph_1024_stream.data")


def read_stream_file(path: str):
    """(V, types u8[n], pairs u32[n, 2])."""
    with open(path, "rb") as f:
        d = f.read()
    V, n = struct.unpack_from("<IQ", d, 0)
    rec = np.frombuffer(d, np.uint8, count=9 * n, offset=12).reshape(n, 9)
    pairs = rec[:, 1:].copy().view("<u4").reshape(n, 2).astype(np.uint32)
    return V, rec[:, 0].copy(), pairs


def write_stream_file(path: str, V: int, pairs: np.ndarray, types: np.ndarray | None = None) -> None:
    """Writes records in the same format; without `types`, a record is a delete when it toggles an
    edge that is present."""
    p = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
    if types is None:
        present, t = set(), np.zeros(len(p), np.uint8)
        for i, (a, b) in enumerate(p.tolist()):
            e = (min(a, b), max(a, b))
            t[i] = 1 if e in present else 0
            present.symmetric_difference_update({e})
        types = t
    rec = np.empty((len(p), 9), np.uint8)
    rec[:, 0] = types
    rec[:, 1:] = p.astype("<u4").view(np.uint8).reshape(-1, 8)
    with open(path, "wb") as f:
        f.write(struct.pack("<IQ", V, len(p)))
        f.write(rec.tobytes())
