"""The C++ drop-in classes (gpusketch_b200/cpp) driven the way the reference's
tools/cuda_process_stream.cu drives CCGPUSketchAlg: binary stream file -> GraphSketchDriver ->
connected_components(), plus the write_binary checkpoint."""
import hashlib
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from stream_file import write_stream_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "gpusketch_b200", "_build", "cc_dropin_demo")


@pytest.mark.gpu
def test_cpp_dropin_driver_matches_reference(tmp_path, golden_dir):
    assert os.path.exists(DEMO), "build() compiles the C++ drop-in demo"
    case = [c for c in json.load(open(os.path.join(golden_dir, "ref_digests.json"))) if c["name"] == "multiples_1024"][0]
    pairs = np.load(os.path.join(golden_dir, "multiples_1024_stream.npy"))
    stream = str(tmp_path / "multiples.data")
    ck = str(tmp_path / "ck.bin")
    write_stream_file(stream, 1024, pairs)
    out = subprocess.run([DEMO, stream, str(int(case["seed"])), ck, "3"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("num_cc=")]
    assert len(lines) == 3
    assert lines[-1].startswith("num_cc=78 ")
    data = open(ck, "rb").read()
    assert hashlib.sha256(data[20:]).hexdigest() == case["sketch_sha256"]


def test_stream_file_format_roundtrip(tmp_path):
    """The writer above produces the format the reference's fixture uses (9-byte records)."""
    pairs = np.array([[1, 2], [2, 1], [3, 4]], np.uint32)
    p = str(tmp_path / "s.data")
    write_stream_file(p, 8, pairs)
    d = open(p, "rb").read()
    assert len(d) == 12 + 9 * 3
    assert struct.unpack_from("<IQ", d, 0) == (8, 3)
    assert [d[12 + 9 * k] for k in range(3)] == [0, 1, 0]
