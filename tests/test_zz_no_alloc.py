"""xt_count_device_static: the count for callers that cannot allocate device
memory while they run (their device memory is all reserved by another pool, or
they run under a hard memory quota, or must never wait on the allocator).

Through the C ABI, its count must equal the allocating entry point's
(xt_count_device) on the same device CSR, exactly, on two calls in a row (the
fixed scratch array keeps the previous call's contents, so the second call
shows the clearing works), and the device's free memory must not move while
it runs. This file is named so that pytest collects it last.
"""
import numpy as np
import pytest

import oracle
import xxtric_b200 as xt
from conftest import load_fixtures, load_golden

pytestmark = pytest.mark.gpu

GOLDEN = load_golden()
FIX = load_fixtures()


def device_csr(torch, off, tails):
    return torch.from_numpy(off).cuda(), torch.from_numpy(tails).cuda()


def canon(name):
    f = GOLDEN[name]
    return oracle.canon_csr(f["nv"], FIX[name + "_src"].astype(np.int64), FIX[name + "_dst"].astype(np.int64))


@pytest.mark.parametrize("name", ["amazon0302", "chunglu14", "rmat14", "k64", "iso_tail"])
def test_static_scratch_matches_allocating_entry_point(name):
    import torch
    off, tails = canon(name)
    nv = len(off) - 1
    d_off, d_t = device_csr(torch, off, tails)
    stream = torch.cuda.current_stream().cuda_stream
    ref = torch.zeros(1, dtype=torch.int64, device="cuda")
    xt.count_device(nv, d_off, d_t, ref, stream=stream)
    out = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    xt.count_device_static(nv, d_off, d_t, out, stream=stream)  # first call on the device: set-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        out.fill_(-7)
        xt.count_device_static(nv, d_off, d_t, out, stream=stream)
        torch.cuda.synchronize()
        assert int(out.item()) == int(ref.item()) == GOLDEN[name]["triangles"]
    assert torch.cuda.mem_get_info()[0] == free0
    xt.count_device_static(nv, d_off, d_t, out, accumulate=True, stream=stream)
    torch.cuda.synchronize()
    assert int(out.item()) == 2 * GOLDEN[name]["triangles"]


def test_static_scratch_size_limit_and_bad_input():
    import torch
    d = torch.zeros(8, dtype=torch.int64, device="cuda")
    with pytest.raises(xt.XtError) as e:
        xt.count_device_static(8389089, d, d, d)
    assert e.value.status == xt.XT_ERR_OVERFLOW
    # a row whose neighbour lacks the back edge: reported, not miscounted silently
    off = torch.tensor([0, 2, 4, 6], dtype=torch.int64, device="cuda")  # the triangle 0-1-2
    tails = torch.tensor([1, 2, 0, 2, 0, 1], dtype=torch.int64, device="cuda")
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    # rows: 0 -> {2}, 1 -> {0, 2}, 2 -> {0, 1}: row 0 lacks the back edge to 1
    off2 = torch.tensor([0, 1, 3, 5], dtype=torch.int64, device="cuda")
    tails2 = torch.tensor([2, 0, 2, 0, 1], dtype=torch.int64, device="cuda")
    with pytest.raises(xt.XtError) as e:
        xt.count_device_static(3, off2, tails2, out, stream=torch.cuda.current_stream().cuda_stream)
    assert e.value.status == xt.XT_ERR_INVALID
    # rows this entry cannot repair (it has no room to sort): out of order, a
    # repeated id, the row's own id, an id past nv. Its input check rejects
    # them before any pass indexes memory with them.
    bad = [([0, 2, 4, 6], [2, 1, 0, 2, 0, 1]),   # row 0 out of order
           ([0, 3, 5, 7], [1, 1, 2, 0, 2, 0, 1]),  # row 0 repeats 1
           ([0, 3, 5, 7], [0, 1, 2, 0, 2, 0, 1]),  # row 0 holds 0
           ([0, 2, 4, 6], [1, 5, 0, 2, 0, 1])]     # id 5 with nv = 3
    for o, t in bad:
        with pytest.raises(xt.XtError) as e:
            xt.count_device_static(3, torch.tensor(o, dtype=torch.int64, device="cuda"),
                                   torch.tensor(t, dtype=torch.int64, device="cuda"), out,
                                   stream=torch.cuda.current_stream().cuda_stream)
        assert e.value.status == xt.XT_ERR_INVALID, (o, t)
    # a valid graph afterwards still counts
    xt.count_device_static(3, off, tails, out, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(out.item()) == 1


def test_static_scratch_asymmetric_rows_leave_the_counter_alone():
    """An edge listed in one of its two rows only is rejected in either
    direction, and the output counter keeps its value on every error, in the
    overwrite and the accumulate forms."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    cases = [
        # row 0 lists 1 (1 > 0) but row 1 lacks 0: the upper-row direction
        ([0, 2, 3, 5], [1, 2, 2, 0, 1]),
        # row 1 lists 0 (0 < 1) but row 0 lacks 1: the lower-row direction
        ([0, 1, 3, 5], [2, 0, 2, 0, 1]),
    ]
    for o, t in cases:
        d_o = torch.tensor(o, dtype=torch.int64, device="cuda")
        d_t = torch.tensor(t, dtype=torch.int64, device="cuda")
        for acc in (False, True):
            out = torch.full((1,), 41, dtype=torch.int64, device="cuda")
            with pytest.raises(xt.XtError) as e:
                xt.count_device_static(3, d_o, d_t, out, accumulate=acc, stream=stream)
            assert e.value.status == xt.XT_ERR_INVALID, (o, t, acc)
            torch.cuda.synchronize()
            assert int(out.item()) == 41, (o, t, acc)
    # a bad row (out of order) leaves the counter alone too
    out = torch.full((1,), 41, dtype=torch.int64, device="cuda")
    with pytest.raises(xt.XtError):
        xt.count_device_static(3, torch.tensor([0, 2, 4, 6], dtype=torch.int64, device="cuda"),
                               torch.tensor([2, 1, 0, 2, 0, 1], dtype=torch.int64, device="cuda"), out,
                               accumulate=True, stream=stream)
    torch.cuda.synchronize()
    assert int(out.item()) == 41
