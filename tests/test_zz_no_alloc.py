"""The allocation-free induce entry point gives exactly what the regular one
gives.

lg_induce_sumcheck_poly_noalloc exists for callers that cannot allocate
device memory (their GPU memory belongs to another allocator, or they must
not risk the device-wide synchronisation of cudaMalloc / cudaFree).  It
takes only caller buffers plus a fixed scratch array inside the library.
This file checks it bit-for-bit against lg_induce_sumcheck_poly, on two
calls in a row whose sizes differ (the second call must not see anything
the first left in the shared scratch), and that sizes past the scratch
limit are refused without queuing work.  It is collected last so a run that
stops at the first failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(rng, n, nch, nrows=148):
    rows = rng.integers(0, 2**32, size=(nrows, 1 << nch), dtype=np.uint64).astype(np.uint32)
    q = np.sort(rng.choice(4 << n, size=nrows, replace=False)).astype(np.uint64)
    ch = rng.integers(0, 2**32, size=nch, dtype=np.uint64).astype(np.uint32)
    alpha = int(rng.integers(0, 2**32))
    return rows, q, ch, alpha


def _noalloc(lg, n, rows, q, ch, alpha, garbage=0x5A5A5A5A):
    import torch

    rows_d = torch.from_numpy(rows.reshape(-1).view(np.int32)).cuda()
    q_d = torch.from_numpy(q.view(np.int64)).cuda()
    out_d = torch.full((1 << n,), garbage, dtype=torch.int32, device="cuda")
    sum_d = torch.full((1,), garbage, dtype=torch.int32, device="cuda")
    ch = np.ascontiguousarray(ch, dtype=np.uint32)
    torch.cuda.synchronize()
    st = lg.lib.lg_induce_sumcheck_poly_noalloc(None, n, rows_d.data_ptr(), rows.shape[0], ch.ctypes.data, ch.size,
                                                 q_d.data_ptr(), alpha, out_d.data_ptr(), sum_d.data_ptr())
    torch.cuda.synchronize()
    return st, out_d, sum_d


def test_noalloc_matches_regular_entry_point_twice(lg, ctx):
    import torch

    rng = np.random.default_rng(2026)
    # a large call, then a smaller one: the second must not pick up the
    # scratch contents the first left behind
    for n, nch in ((16, 6), (9, 4)):
        rows, q, ch, alpha = _inputs(rng, n, nch)
        want_basis, want_sum = lg.induce_sumcheck_poly(n, rows, ch, q, alpha, ctx)
        st, out_d, sum_d = _noalloc(lg, n, rows, q, ch, alpha)
        assert st == 0, lg.STATUS.get(st, st)
        assert torch.equal(out_d, want_basis)
        assert int(sum_d.cpu().numpy().view(np.uint32)[0]) == want_sum


def test_noalloc_on_a_caller_stream_runs_after_the_callers_work(lg, ctx):
    # Work queued on the caller's stream runs behind what the caller queued
    # there before: a write of garbage into the outputs, queued just ahead
    # of the call on the same stream, must be overwritten by the result.
    import torch

    rng = np.random.default_rng(99)
    n, nch = 14, 6
    rows, q, ch, alpha = _inputs(rng, n, nch)
    want_basis, want_sum = lg.induce_sumcheck_poly(n, rows, ch, q, alpha, ctx)
    rows_d = torch.from_numpy(rows.reshape(-1).view(np.int32)).cuda()
    q_d = torch.from_numpy(q.view(np.int64)).cuda()
    out_d = torch.zeros((1 << n,), dtype=torch.int32, device="cuda")
    sum_d = torch.zeros((1,), dtype=torch.int32, device="cuda")
    ch = np.ascontiguousarray(ch, dtype=np.uint32)
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        torch.cuda._sleep(1 << 20)  # keeps the stream busy while the call is queued
        out_d.fill_(0x33333333)
        sum_d.fill_(0x33333333)
    st = lg.lib.lg_induce_sumcheck_poly_noalloc(s.cuda_stream, n, rows_d.data_ptr(), rows.shape[0], ch.ctypes.data,
                                                 ch.size, q_d.data_ptr(), alpha, out_d.data_ptr(), sum_d.data_ptr())
    assert st == 0
    s.synchronize()
    assert torch.equal(out_d, want_basis)
    assert int(sum_d.cpu().numpy().view(np.uint32)[0]) == want_sum


def test_noalloc_refuses_sizes_past_its_scratch(lg):
    import torch

    rng = np.random.default_rng(7)
    rows, q, ch, alpha = _inputs(rng, 21, 2)
    st, out_d, _ = _noalloc(lg, 21, rows, q, ch, alpha, garbage=7)
    assert st == 9  # LG_ERR_EXCEEDS_STATIC_SCRATCH
    assert bool((out_d == 7).all())  # nothing was queued
    rows, q, ch, alpha = _inputs(rng, 8, 2, nrows=300)
    st, _, _ = _noalloc(lg, 8, rows, q, ch, alpha)
    assert st == 9
