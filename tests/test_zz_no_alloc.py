"""sp_dot_noalloc, the allocation-free dot product, against the existing sp_dot.

It is for callers that cannot allocate device memory at the point of the call
(inside stream capture, under their own pool allocator, in a loop that must not
synchronise on cudaMalloc/cudaFree): it takes raw device pointers, allocates
nothing, and keeps its partial sums in a static device array of fixed size. This
file is named so pytest collects it last; it must pass alone in a fresh process
and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import xorshift_vector

pytestmark = pytest.mark.gpu

SP_OK, SP_ERR_TOO_LARGE = 0, 3
MAX_N = 67108864  # SP_NOALLOC_DOT_MAX_N


def close(a, b):
    """The scalar tolerance of the parity tests (crates/saddlepoint-cuda/tests/ops.rs:41-44)."""
    return abs(a - b) / (1.0 + max(abs(a), abs(b))) < 1e-11


def test_dot_noalloc_matches_sp_dot_on_two_calls(gpu_backend):
    import torch

    import saddlepoint_b200 as sp

    lib = sp.library()
    stream = torch.cuda.current_stream()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    for seed, n in ((3, 1_234_567), (4, 300_001)):
        a_h, b_h = xorshift_vector(n, seed), xorshift_vector(n, seed + 100)
        a = torch.from_numpy(a_h).cuda()
        b = torch.from_numpy(b_h).cuda()
        rc = lib.sp_dot_noalloc(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                C.c_void_p(stream.cuda_stream))
        assert rc == SP_OK
        stream.synchronize()
        got = float(out.item())
        # the existing entry point, through its own context and vectors
        want = gpu_backend.dot(gpu_backend.upload(a_h), gpu_backend.upload(b_h))
        assert close(got, want), (n, got, want)
        assert abs(got - float(np.dot(a_h, b_h))) <= 1e-12 * (1.0 + abs(got))


def test_dot_noalloc_rejects_lengths_beyond_its_scratch(gpu_backend):
    import torch

    import saddlepoint_b200 as sp

    lib = sp.library()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    x = torch.ones(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(x.data_ptr())
    assert lib.sp_dot_noalloc(p, p, MAX_N + 1, C.c_void_p(out.data_ptr()), None) == SP_ERR_TOO_LARGE
    assert lib.sp_dot_noalloc(p, p, 8, C.c_void_p(out.data_ptr()), None) == SP_OK
    torch.cuda.synchronize()
    assert float(out.item()) == 8.0


def test_dot_noalloc_at_its_maximum_length(gpu_backend):
    """n = SP_NOALLOC_DOT_MAX_N fills every partial-sum slot of the static array. The
    entries (1 and (k mod 7) - 3) make every partial sum an exact integer, so the result
    equals the float64 value of the exact sum whatever the order of the additions."""
    import torch

    import saddlepoint_b200 as sp

    lib = sp.library()
    n = MAX_N
    a = torch.ones(n, dtype=torch.float64, device="cuda")
    b = (torch.arange(n, dtype=torch.int64, device="cuda") % 7 - 3).to(torch.float64)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    exact = sum((k % 7) - 3 for k in range(n % 7))  # whole periods of 7 sum to zero
    for _ in range(2):
        rc = lib.sp_dot_noalloc(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                C.c_void_p(stream.cuda_stream))
        assert rc == SP_OK
        stream.synchronize()
        assert float(out.item()) == float(exact)
    del a, b
    torch.cuda.empty_cache()
