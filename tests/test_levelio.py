"""CPU round trip of the level<L>_*.bin format (Python side; the C++ side is
exercised by tests/cpp/test_host.cpp)."""
import numpy as np


def test_level_files_roundtrip(tmp_path):
    from fem_b200 import levelio
    p = levelio.level_paths(str(tmp_path), 2)
    mats = [np.arange(64) % 2, np.ones(8, dtype=np.int32), np.zeros(0, dtype=np.int32)]
    levelio.write_vectors(p["matAssignments"], mats)
    back = levelio.read_vectors(p["matAssignments"])
    assert len(back) == 3 and all(np.array_equal(a, b) for a, b in zip(mats, back))
    params = np.linspace(0, 1, 12, dtype=np.float32)
    levelio.write_vector(p["params"], params)
    assert np.array_equal(levelio.read_vector(p["params"]), params)
    C = np.arange(72, dtype=np.float64).reshape(2, 6, 6)
    levelio.tensors_to_level_file(p["elasticityTensors"], C)
    t = levelio.read_vector(p["elasticityTensors"])
    assert t.size == 42 and t[1] == C[0, 1, 0] and t[21] == C[1, 0, 0]
    # byte layout: int32 count then raw little-endian values
    raw = open(p["params"], "rb").read()
    assert int.from_bytes(raw[:4], "little") == 12 and len(raw) == 4 + 48
