"""aed_dot_noalloc, the dot product that allocates nothing (needs a GPU).

Some callers cannot let a library allocate device memory: applications whose
device memory belongs to another allocator (a framework's caching allocator,
a fixed arena handed to a simulation code) and latency-critical loops that
cannot pay for cudaMalloc/cudaFree.  aed_dot_noalloc keeps its scratch in a
fixed array inside libaed.so; the caller passes only the inputs and the
output.  This test calls it through the C ABI twice in a row and checks each
result against aed_dot on the same vectors: it forms the same chunks and sums
them in the same order, so the two must agree bit for bit.  The lengths cover
one pass of the grid over the chunks (L = 16, 24) and several passes (L = 26:
2,539 chunks against a grid of 8 CTAs per SM; the 6x5 square lattice's
155,117,520 elements, near the 268,435,456 the scratch holds).  It runs alone
or after the other tests.
"""

import ctypes

import numpy as np
import pytest

import alps_b200 as ed

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 65536 * 4096


def chain(L):
    return [(i, (i + 1) % L, 1.0, 1.0) for i in range(L)]


def square6x5():
    out = []
    for x in range(6):
        for y in range(5):
            s = x * 5 + y
            out.append((s, x * 5 + (y + 1) % 5, 1.0, 1.0))
            out.append((s, ((x + 1) % 6) * 5 + y, 1.0, 1.0))
    return out


@pytest.mark.parametrize("L,prec", [(16, ed.FP64), (24, ed.FP64), (24, ed.FP32), (26, ed.FP32), (26, ed.FP64),
                                    (30, ed.FP32)])
def test_dot_noalloc_matches_aed_dot_twice(L, prec):
    import torch

    bonds = square6x5() if L == 30 else chain(L)
    ham = ed.Hamiltonian(L, L // 2, bonds, precision=prec)
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
    assert got[0] == ref and got[1] == ref, (got, ref)
    x.free()
    y.free()
    ham.close()


def test_dot_noalloc_empty_is_zero():
    import torch

    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    rc = ed.lib().aed_dot_noalloc(None, None, 0, ed.FP64, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == ed.OK, ed.lib().aed_last_error()
    torch.cuda.synchronize()
    assert out.item() == 0.0


def test_dot_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    ham = ed.Hamiltonian(8, 4, chain(8))
    x = ham.new_vector()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = ed.lib().aed_dot_noalloc(x.ptr, x.ptr, MAX_ELEMENTS + 1, ed.FP64, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == ed.ERR_INVALID
    assert b"exceeds the static scratch" in ed.lib().aed_last_error()
