"""kmy_conserved_sums_noalloc: the sums for callers that cannot allocate device
memory (GPU).

The entry point works on caller-owned device arrays and keeps its partial
sums in a static device array, so a framework that owns all device memory, or
code that may not allocate, can still take the FP64 conservation sums.  This
file is collected last so that a run stopping at the first failure has
already run every other test; it also passes when run alone in a fresh
process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONS = [("dens", 0), ("momentum", 0), ("momentum", 1), ("momentum", 2), ("ener", 0)]
TOL = 1e-14


def _ints(v):
    return (ctypes.c_int * 3)(*v)


def test_noalloc_sums_match_context_sums_twice(kmy_lib):
    import torch

    import kamayan_b200 as K
    from kamayan_b200 import configs

    # 128^3 interior cells: more than the kernel's 151,552 threads, so each
    # thread's grid-stride loop and its compensated sum run several times
    s = K.Solver(configs.kh_3d(n=128, nb=32))
    s.pgen("kelvin_helmholtz")
    s.step()
    assert s.info.nblocks * 32 ** 3 > 4 * 592 * 256
    ref = s.conserved_sums()
    inf = s.info
    vol = inf.dx[0] * inf.dx[1] * inf.dx[2]
    host = np.ascontiguousarray(np.stack([s.export(v, c) for v, c in CONS]))
    # the test allocates the caller's buffers; the entry point allocates nothing
    cons = torch.from_numpy(host).cuda()
    out = torch.empty(len(CONS), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    g = [inf.nghost if d < inf.ndim else 0 for d in range(3)]
    args = (len(CONS), inf.nblocks, _ints(list(inf.ncells_pad)), _ints(list(inf.nx)), _ints(g), vol)
    for call in range(2):
        out.fill_(float("nan"))
        rc = kmy_lib.kmy_conserved_sums_noalloc(ctypes.c_void_p(cons.data_ptr()), *args,
                                                ctypes.c_void_p(out.data_ptr()),
                                                ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=TOL, atol=1e-16,
                                   err_msg=f"call {call + 1}")
    # a changed input is seen by the next call (no state carried between calls)
    cons[0].mul_(2.0)
    rc = kmy_lib.kmy_conserved_sums_noalloc(ctypes.c_void_p(cons.data_ptr()), *args,
                                            ctypes.c_void_p(out.data_ptr()),
                                            ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert out[0].item() == pytest.approx(2.0 * ref[0], rel=TOL)


def test_noalloc_rejects_sizes_beyond_scratch(kmy_lib):
    import torch

    cons = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = kmy_lib.kmy_conserved_sums_noalloc(ctypes.c_void_p(cons.data_ptr()), 9, 1,
                                            _ints([1, 1, 1]), _ints([1, 1, 1]), _ints([0, 0, 0]),
                                            1.0, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1  # KMY_ERR_BAD_PARAM
