"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on a CPU-only machine."""
import csv
import gzip
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
NETLIB = os.path.join(GOLDEN, "netlib")

# Instance lists of the reference's Netlib regression (crates/saddlepoint-cpu/tests/netlib.rs:13-26).
QUICK = ["afiro", "adlittle", "israel", "sctest", "shell", "etamacro", "standata", "standgub", "standmps",
         "forest6", "woodinfe"]
SLOW = ["25fv47", "80bau3b", "scrs8", "stair", "perold"]
KNOWN_HARD = ["greenbea", "klein1"]
TOL = 1e-6


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running")


def netlib_bytes(name: str) -> bytes:
    with gzip.open(os.path.join(NETLIB, f"{name}.mps.gz"), "rb") as f:
        return f.read()


def netlib_reference():
    """data/netlib/reference.csv: HiGHS 1.15.1 status and objective per instance."""
    out = {}
    with open(os.path.join(NETLIB, "reference.csv")) as f:
        for r in csv.DictReader(f):
            out[r["name"]] = (r["status"], float(r["objective"]) if r["objective"] else None)
    return out


_cache = {}


def netlib_lp(name: str):
    """The Netlib LP read by the oracle's MPS reader (crates/saddlepoint-io/src/lib.rs:59-309)."""
    if name not in _cache:
        import oracle

        _cache[name] = oracle.read_mps(netlib_bytes(name), name)
    return _cache[name]


def xorshift_vector(length: int, seed: int) -> np.ndarray:
    """Deterministic values in [-2, 2], every fifth one zero (crates/saddlepoint-cuda/tests/ops.rs:29-39)."""
    mask = (1 << 64) - 1
    s = ((seed * 0x9E3779B97F4A7C15) & mask) | 1
    out = np.empty(length)
    for i in range(length):
        s ^= (s << 13) & mask
        s ^= s >> 7
        s ^= (s << 17) & mask
        out[i] = 0.0 if i % 5 == 0 else (s >> 11) / float(1 << 53) * 4.0 - 2.0
    return out


@pytest.fixture(scope="session")
def gpu_backend():
    """The CUDA backend on device 0; a GPU test fails (never skips) when it cannot be opened."""
    import saddlepoint_b200 as sp

    b = sp.CudaBackend(0)
    yield b
    b.close()
