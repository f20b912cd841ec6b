"""aed_dot_noalloc, the dot product that allocates nothing (needs a GPU).

Some callers cannot let a library allocate device memory: applications whose
device memory belongs to another allocator (a framework's caching allocator,
a fixed arena handed to a simulation code) and latency-critical loops that
cannot pay for cudaMalloc/cudaFree.  aed_dot_noalloc keeps its scratch in a
fixed array inside libaed.so; the caller passes only the inputs and the
output.  This test calls it through the C ABI twice in a row and checks each
result against aed_dot on the same vectors, with the tolerance the other
vector tests use (it uses the same chunks and summation order, so the bits
agree in practice).  It runs alone or after the other tests.
"""

import ctypes

import numpy as np
import pytest

import alps_b200 as ed

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 65536 * 4096


def chain(L):
    return [(i, (i + 1) % L, 1.0, 1.0) for i in range(L)]


@pytest.mark.parametrize("L,prec", [(16, ed.FP64), (24, ed.FP64), (24, ed.FP32)])
def test_dot_noalloc_matches_aed_dot_twice(L, prec):
    import torch

    ham = ed.Hamiltonian(L, L // 2, chain(L), precision=prec)
    x, y = ham.new_vector(), ham.new_vector()
    ham.fill_random(x, 11)
    ham.fill_random(y, 12)
    ref = ham.dot(x, y)  # aed_dot; returns after the handle's stream is done
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    for k in range(2):
        rc = ed.lib().aed_dot_noalloc(x.ptr, y.ptr, ham.dim, prec, ctypes.c_void_p(out.data_ptr() + 8 * k), None)
        assert rc == ed.OK, ed.lib().aed_last_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.all(np.abs(got - ref) <= 1e-12 * abs(ref)), (got, ref)


def test_dot_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    ham = ed.Hamiltonian(8, 4, chain(8))
    x = ham.new_vector()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = ed.lib().aed_dot_noalloc(x.ptr, x.ptr, MAX_ELEMENTS + 1, ed.FP64, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == ed.ERR_INVALID
    assert b"exceeds the static scratch" in ed.lib().aed_last_error()
