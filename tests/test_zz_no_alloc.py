"""fmmb_direct_noalloc_dev: the FP64 direct sums for callers that cannot call cudaMalloc (an
application whose device memory is held by its own pool, or a loop that must not pay
cudaMalloc's implicit synchronisation). Its partial sums live in a fixed 4 MiB array compiled
into the library instead of a per-call allocation; the results must equal those of
fmmb_direct_dev (the allocating entry point) within the tolerance of the direct-sum test,
on two calls in a row (the second reuses the array the first left behind)."""
import ctypes as C

import numpy as np
import pytest

from helpers import mrd

pytestmark = pytest.mark.gpu


def _call(fmmb, name, ctx, s, t, g, sel, pot, grad):
    fn = getattr(fmmb.lib(), name)
    p = lambda x: None if x is None else C.c_void_p(x.data_ptr())
    rc = fn(ctx._h, p(s), p(t), s.shape[0], p(g), p(sel), g.shape[0], p(pot), p(grad))
    return rc


def test_no_alloc_direct_matches_the_allocating_entry_point(fmmb):
    import torch
    ctx = fmmb.default_context()
    rng = np.random.default_rng(5)
    n = 20000
    src = torch.from_numpy(rng.random((n, 3))).cuda()
    tau = torch.from_numpy(rng.standard_normal(n)).cuda()
    # (targets, at the sources, with the gradient): the split counts of both entry points agree
    # for the first two; 131,072 is the largest nt (one source range in the scratch), 100 targets
    # hit the cap of 32 ranges (fmmb_direct_dev takes more), and one call has no gradient output
    for nt, self_, with_grad in ((3000, True, True), (4096, False, True), (1 << 17, False, True), (100, True, True),
                                 (2000, False, False)):
        sel = torch.from_numpy(np.sort(rng.choice(n, nt, replace=False)).astype(np.int64)).cuda() if self_ else None
        tgt = src[sel].contiguous() if self_ else torch.from_numpy(rng.random((nt, 3))).cuda()
        ref_p = torch.zeros(nt, dtype=torch.float64, device="cuda")
        ref_g = torch.zeros((nt, 3), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert _call(fmmb, "fmmb_direct_dev", ctx, src, tau, tgt, sel, ref_p, ref_g) == 0
        for _ in range(2):                               # two calls in a row share the scratch array
            pot = torch.full((nt,), np.nan, dtype=torch.float64, device="cuda")
            grad = torch.full((nt, 3), np.nan, dtype=torch.float64, device="cuda") if with_grad else None
            torch.cuda.synchronize()
            assert _call(fmmb, "fmmb_direct_noalloc_dev", ctx, src, tau, tgt, sel, pot, grad) == 0
            assert fmmb.lib().fmmb_ctx_synchronize(ctx._h) == 0
            assert mrd(pot.cpu().numpy(), ref_p.cpu().numpy()) < 1e-13, nt
            if with_grad:
                assert mrd(grad.cpu().numpy(), ref_g.cpu().numpy()) < 1e-13, nt


def test_no_alloc_direct_rejects_sizes_beyond_its_scratch(fmmb):
    import torch
    ctx = fmmb.default_context()
    src = torch.zeros((10, 3), dtype=torch.float64, device="cuda")
    tau = torch.zeros(10, dtype=torch.float64, device="cuda")
    nt = (1 << 17) + 1                                   # one target above the 131,072 maximum
    tgt = torch.zeros((nt, 3), dtype=torch.float64, device="cuda")
    pot = torch.zeros(nt, dtype=torch.float64, device="cuda")
    rc = _call(fmmb, "fmmb_direct_noalloc_dev", ctx, src, tau, tgt, None, pot, None)
    assert rc == fmmb.FMMB_OK + 1
    assert b"at most 131072 targets" in fmmb.lib().fmmb_last_error()
