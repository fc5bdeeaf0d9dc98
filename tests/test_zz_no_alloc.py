"""karam_eval_stamp_noalloc: evaluation + stamping into caller-owned device
buffers with no device allocation inside the call (for callers whose GPU memory
belongs to their own pool allocator, or who cannot afford the device
synchronisation of cudaMalloc). Its results must equal karam_eval_stamp's,
call after call, although every call reuses the library's one fixed scratch
array. The test allocates its own buffers with torch; the entry point does not.
Kept in a file of its own, collected last."""
import ctypes as C

import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_noalloc_matches_eval_stamp_twice(product, ctx, prec):
    import torch
    nl = circuits.config2()
    ni = 3
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(circuits.mc_instances(nl, ni))
    n, nnz = prob.n, prob.info["nnz"]
    lib = product.lib()
    rng = np.random.default_rng(11)
    for call in range(2):
        v = rng.uniform(-0.2, 2.0, size=(ni, n))
        jac_ref, f_ref = prob.eval_stamp(v, prec)
        d_v = torch.tensor(v, dtype=torch.float64, device="cuda")
        d_jac = torch.full((ni, nnz), np.nan, dtype=torch.float64, device="cuda")
        d_f = torch.full((ni, n), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.karam_eval_stamp_noalloc(prob.h, prec, C.c_void_p(d_v.data_ptr()),
                                          C.c_void_p(d_jac.data_ptr()), C.c_void_p(d_f.data_ptr()))
        assert rc == A.KARAM_OK, lib.karam_last_error(ctx.h).decode()
        jac, f = d_jac.cpu().numpy(), d_f.cpu().numpy()
        # the same kernel on the same inputs: identical values
        assert np.array_equal(jac, jac_ref), (call, np.max(np.abs(jac - jac_ref)))
        assert np.array_equal(f, f_ref), (call, np.max(np.abs(f - f_ref)))


def test_noalloc_rejects_problems_beyond_its_scratch(product, ctx):
    import torch
    nl = circuits.config2()
    prob = product.Problem(ctx, nl, max_instances=4096)  # needs ~60 MB of scratch
    d = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = C.c_void_p(d.data_ptr())
    rc = product.lib().karam_eval_stamp_noalloc(prob.h, A.PREC_FP64, p, p, p)
    assert rc == A.KARAM_E_INVALID
    assert "scratch" in product.lib().karam_last_error(ctx.h).decode()
