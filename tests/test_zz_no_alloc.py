"""aster_energy_noalloc: the energy entry point for callers that cannot
allocate device memory (codes that own all GPU memory through their own pool,
loops that must not allocate mid-run). It takes the caller's device arrays and
keeps its scratch in a fixed array inside the library.

Checked through the C ABI against the context-based aster_energy on two calls
in a row per size (the shared scratch keeps the previous call's contents; the
second call must not depend on them). The sizes run small, large, then small
again, so a small call also follows a large one that filled more of the
scratch; the last size runs on a stream of its own (the call queues its work
there and returns). Tolerance: relative 1e-12 on the energy, absolute 1e-14 on
the momentum (the two paths run the same kernels).

This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

from aster_b200 import gen
from aster_b200.api import CParams, Context, Params, load_library

pytestmark = pytest.mark.gpu

ASTER_ERR_TOO_LARGE = 10
MAX_N = 65536 * 256


def _entry():
    f = load_library().aster_energy_noalloc
    f.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(CParams), ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("ref_form", [0, 1])
def test_noalloc_energy_matches_context_energy(ref_form):
    import torch

    f = _entry()
    dev = torch.device("cuda", 0)
    side = torch.cuda.Stream(device=dev)
    for n, seed, stream in ((1000, 11, None), (70001, 12, None), (1000, 13, side)):
        pos, vel, m = gen.plummer(n, seed)
        p = Params(eps2=1e-4)
        with Context(0) as ctx:
            ctx.upload(pos, vel, m)
            e_ref, mom_ref = ctx.energy(p, ref_form=bool(ref_form))
        pm = torch.tensor(np.c_[pos, m], dtype=torch.float64, device=dev).contiguous()
        v4 = torch.tensor(np.c_[vel, np.zeros(n)], dtype=torch.float64, device=dev).contiguous()
        out = torch.empty(4, dtype=torch.float64, device=dev)
        cp = p.c_struct()
        for _ in range(2):
            out.fill_(float("nan"))
            torch.cuda.synchronize()
            handle = stream.cuda_stream if stream is not None else None
            st = f(n, pm.data_ptr(), v4.data_ptr(), ctypes.byref(cp), ref_form, out.data_ptr(), handle)
            assert st == 0
            if stream is not None:
                stream.synchronize()  # only the stream the work was queued on
            else:
                torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert abs(got[0] - e_ref) <= 1e-12 * abs(e_ref), (got[0], e_ref)
            np.testing.assert_allclose(got[1:], mom_ref, rtol=0, atol=1e-14)


def test_noalloc_energy_rejects_sizes_beyond_its_scratch():
    f = _entry()
    cp = Params().c_struct()
    # rejected before any device access, so placeholder aligned addresses do
    st = f(MAX_N + 1, 256, 256, ctypes.byref(cp), 0, 256, None)
    assert st == ASTER_ERR_TOO_LARGE
