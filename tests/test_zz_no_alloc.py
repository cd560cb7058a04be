"""The refinement entry point that allocates nothing (cp_refine_boxes_static).

It exists for callers that cannot let a library allocate device memory -- programs
that route every allocation through their own pool, and latency-critical loops
that cannot afford cudaMalloc's implicit synchronisation -- and keeps its scratch
in a fixed array compiled into the library.  These tests call it through the C
ABI and check that it reports exactly what the allocating entry point
cp_refine_boxes reports for the same seeds, on two calls in a row (the second
call runs on the array the first one left behind).  This file is collected last
so that a failure here does not stop the other GPU tests.
"""
import ctypes

import numpy as np
import pytest

from tests import boxgen

pytestmark = pytest.mark.gpu


def _seeds(cp, family, sizes):
    total = int(np.prod(sizes))
    lo, hi, vis = cp.lattice_boxes(family, boxgen.LAMBDA, sizes, np.arange(total), visited=True)
    import torch

    depth = torch.where(vis != 0, 0, 255).to(torch.uint8)
    return lo, hi, depth


def _static_call(cp, family, lo, hi, depth, precision, policy, max_depth):
    import torch

    L = cp.lib()
    cp._declare_handle(L)
    r = cp.RefineReport()
    st = L.cp_refine_boxes_static(family, precision, policy, max_depth, ctypes.c_void_p(lo.data_ptr()),
                                  ctypes.c_void_p(hi.data_ptr()), ctypes.c_void_p(depth.data_ptr()), lo.shape[1],
                                  ctypes.byref(r), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, r.as_dict()


@pytest.mark.parametrize("family,precision,policy", [(3, 0, 2), (0, 0, 1), (5, 1, 2), (4, 0, 0)])
def test_static_scratch_matches_allocating_entry(cp, family, precision, policy):
    dims = boxgen.DIMS[family]
    lo, hi, depth = _seeds(cp, family, [16, 8, 8, 4][:dims])
    max_depth = 6 if policy != 0 else 2
    p = cp.Prover(0)
    want = p.refine_boxes(family, lo, hi, depth=depth, precision=precision, policy=policy, max_depth=max_depth)
    p.close()
    keys = ("evaluated", "verdicts", "unresolved", "clipped", "fp32_decided", "per_depth")
    for _ in range(2):
        st, got = _static_call(cp, family, lo, hi, depth, precision, policy, max_depth)
        assert st == 0, cp.lib().cp_last_error_string()
        for k in keys:
            assert got[k] == want[k], (k, got[k], want[k])


def test_static_scratch_rejects_oversize(cp):
    import torch

    n = cp.STATIC_MAX_SEEDS + 1
    lo = torch.zeros((4, n), dtype=torch.float64, device="cuda")
    depth = torch.zeros(n, dtype=torch.uint8, device="cuda")
    st, _ = _static_call(cp, 3, lo, lo, depth, 0, 2, 6)
    assert st == 4  # CP_ERR_CAPACITY
    assert b"at most" in cp.lib().cp_last_error_string()
    st, _ = _static_call(cp, 3, lo[:, :10], lo[:, :10], depth[:10], 0, 2, cp.STATIC_MAX_DEPTH + 1)
    assert st == 4
