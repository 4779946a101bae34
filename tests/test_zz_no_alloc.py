"""The allocation-free FP64 reduction, cbct_reduce_f64_noalloc, on the GPU.

Some callers of this library cannot allocate device memory while they run:
a latency-bound caller sharing the GPU with other work (cudaMalloc may wait
for the whole device to go idle), or a host whose device memory belongs to
another allocator that forbids side allocations.  cbct_reduce_f64 allocates its
partial-sum buffer on first use; cbct_reduce_f64_noalloc keeps the partial
sums in a static device array instead.  This test calls it through the C ABI
and checks it against cbct_reduce_f64 on two calls in a row (a large call,
then a smaller one that reads fewer partials than the first one wrote).

The file is named so that pytest collects it last."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_reduce_matches_allocating_reduce(gtb, cuda):
    import torch
    L = gtb._lib
    stream = torch.cuda.current_stream().cuda_stream
    gen = torch.Generator(device=cuda)
    gen.manual_seed(7)
    for n in (3_000_017, 1_000):
        a = torch.rand(n, generator=gen, device=cuda) - 0.5
        b = torch.rand(n, generator=gen, device=cuda) + 0.25
        a64, b64 = a.double().cpu().numpy(), b.double().cpu().numpy()
        exact = {0: float(np.dot(a64, b64)), 1: float(np.dot(a64, a64)), 2: float(np.abs(a64).sum())}
        for kind in (0, 1, 2):
            ref = torch.zeros(1, dtype=torch.float64, device=cuda)
            got = torch.full((1,), -1.0, dtype=torch.float64, device=cuda)
            L.call("cbct_reduce_f64", kind, a.data_ptr(), b.data_ptr(), n, ref.data_ptr(), stream)
            L.call("cbct_reduce_f64_noalloc", kind, a.data_ptr(), b.data_ptr(), n, got.data_ptr(), stream)
            torch.cuda.synchronize()
            r, g = ref.item(), got.item()
            # same kernel and launch shape: the results agree to the last bit
            assert g == r, (n, kind, g, r)
            assert abs(g - exact[kind]) <= 1e-9 * max(1.0, abs(exact[kind])), (n, kind, g, exact[kind])


def test_noalloc_reduce_rejects_bad_arguments(gtb, cuda):
    import torch
    L = gtb._lib
    a = torch.zeros(16, device=cuda)
    out = torch.zeros(1, dtype=torch.float64, device=cuda)
    st = L.lib().cbct_reduce_f64_noalloc(3, a.data_ptr(), a.data_ptr(), 16, out.data_ptr(), 0)
    assert st == 1
    st = L.lib().cbct_reduce_f64_noalloc(0, a.data_ptr(), None, 16, out.data_ptr(), 0)
    assert st == 1
