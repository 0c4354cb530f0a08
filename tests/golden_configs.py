"""Access to tests/golden/configs.json.gz, the CPU oracle's answers on the
benchmark's full-size workloads (written by tests/golden/make_config_golden.py),
and the matching SHA-256 of device-resident inputs."""
import gzip
import hashlib
import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "configs.json.gz")


def load() -> dict:
    with gzip.open(PATH, "rt") as f:
        return json.load(f)


def entry(name: str) -> dict:
    return load()[name]


def device_sha256(t, chunk: int = 1 << 25) -> str:
    """SHA-256 of a device int64 tensor's little-endian bytes, copied to the
    host in chunks."""
    h = hashlib.sha256()
    flat = t.reshape(-1)
    for i in range(0, flat.numel(), chunk):
        h.update(flat[i:i + chunk].cpu().numpy().view(np.uint64).tobytes())
    return h.hexdigest()


def host_sha256(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()
