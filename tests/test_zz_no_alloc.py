"""ab_square_mul_noalloc: the allocation-free squaring for callers that must
not allocate device memory after start-up (inside a stream capture, under a
fixed memory pool or budget).  Its work buffers are a static device array, so
the output must equal the handle-based ab_square_mul bit for bit, call after
call.  This file is collected last so that a failure here comes after every
other test has run.
"""
import numpy as np
import pytest

import annie_b200 as A
from helpers import pick_N

pytestmark = pytest.mark.gpu


def _device_register(words):
    import torch
    return torch.from_numpy(words.view(np.int32).copy()).to("cuda:0")


@pytest.mark.parametrize("bits", [70000, 262144, 1000000])
def test_noalloc_matches_square_mul_two_calls(bits):
    import torch
    N = pick_N(bits, seed=bits + 5)
    t = A.Transform(N, 3, device=0)
    t.set1()
    t.square_mul(3)
    dev = _device_register(t.read_register(0))
    torch.cuda.synchronize()
    for a in (3, 1):                      # two calls in a row
        t.square_mul(a)                   # existing entry point, on Reg0
        t.square_mul_noalloc(dev.data_ptr(), a)
        t.synchronize()
        torch.cuda.synchronize()
        got = dev.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, t.read_register(0)), "noalloc result differs (a=%d, %d bits)" % (a, bits)


def test_noalloc_rejects_oversize():
    import torch
    # 12M bits: 4 primes x 2^18 words > 2^19 words of static scratch per register
    N = pick_N(12000000, seed=77)
    t = A.Transform(N, 3, device=0)
    assert t.K * t.n > (1 << 19)
    dev = torch.zeros(t.K * t.n, dtype=torch.int32, device="cuda:0")
    with pytest.raises(A.EngineError) as e:
        t.square_mul_noalloc(dev.data_ptr(), 3)
    assert e.value.code == A.AB_E_CAPACITY
