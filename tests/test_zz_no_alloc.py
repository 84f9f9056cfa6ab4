"""The allocation-free error report, d3d_compare_noalloc.

Who needs it: callers that cannot allocate device memory when they ask for
an error report -- a serving loop that already gave all free HBM to its
solve arena, or a host whose allocator policy forbids driver allocations.
The entry point keeps its partial sums in a fixed array inside the
library's device image instead of calling cudaMalloc.

This file is named so that pytest collects it last: if it fails, a run that
stops at the first failure has already run every other test.  It depends on
no state from other tests, so it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import benchmarks_b200 as B

# Same tolerance as the other device-norm test (test_parity_gpu): the two
# entry points sum in different orders, so sums agree to FP64 rounding and
# the maxima agree exactly.
RTOL = 1e-12


def test_noalloc_rejects_oversized_fields_without_a_gpu():
    out = np.zeros(4, np.float64)
    rc = B.lib().d3d_compare_noalloc(
        1, B.F32, 1, B.F32, B.NOALLOC_MAX_ELEMENTS + 1,
        out.ctypes.data_as(B._dp), None)
    assert rc == B.D3D_E_INVALID
    assert "allocation-free limit" in B.lib().d3d_last_error().decode()


@pytest.mark.gpu
def test_noalloc_compare_matches_allocating_compare_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    gen = torch.Generator(device="cuda").manual_seed(99)
    # Two calls in a row on different inputs: the second, smaller call must
    # not see anything left in the shared array by the first.
    cases = [((96, 80, 72), torch.float32, torch.float64),
             ((40, 24, 17), torch.float32, torch.float32)]
    plan = B.Plan(8, 8, 8)  # owns the scratch of the allocating entry point
    for (nx, ny, nz), ta, tb in cases:
        a = torch.rand((nz, ny, nx), device="cuda", generator=gen,
                       dtype=ta) + 0.5
        b = (a.to(tb) + 1e-3 * torch.rand((nz, ny, nx), device="cuda",
                                          generator=gen, dtype=tb))
        got = B.compare_noalloc(a, b)
        exp = plan.compare(a, b)
        np.testing.assert_allclose(got[[0, 3]], exp[[0, 3]], rtol=RTOL)
        assert got[1] == exp[1] and got[2] == exp[2]
        assert got[1] > 0
    # No device memory is taken: free memory is the same before and after
    # a further call (the library has no allocator cache; torch's caching
    # allocator is not involved in the call).
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    got2 = B.compare_noalloc(a, b)
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 == free1
    assert got2[1] == exp[1] and got2[2] == exp[2]
    # A NaN in the field shows in every output, maxima included.
    a.view(-1)[5] = float("nan")
    got3 = B.compare_noalloc(a, b)
    assert np.isnan(got3).all()
    # The call waits for its stream, so a stream under capture is refused
    # before anything is launched, and the capture is left intact.
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    x = torch.zeros(4, device="cuda")
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            x.add_(1.0)
            out = np.zeros(4, np.float64)
            rc = B.lib().d3d_compare_noalloc(
                a.data_ptr(), B.F32, b.data_ptr(), B.F32, 16,
                out.ctypes.data_as(B._dp), ctypes.c_void_p(side.cuda_stream))
    assert rc == B.D3D_E_INVALID
    assert "captured" in B.lib().d3d_last_error().decode()
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
    # Oversized requests are refused before any device work.
    with pytest.raises(B.D3DError) as ei:
        out = np.zeros(4, np.float64)
        B.check(B.lib().d3d_compare_noalloc(
            a.data_ptr(), B.F32, b.data_ptr(), B.F32,
            B.NOALLOC_MAX_ELEMENTS + 1, out.ctypes.data_as(B._dp), None))
    assert ei.value.code == B.D3D_E_INVALID
