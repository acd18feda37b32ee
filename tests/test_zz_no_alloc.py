"""The allocation-free right-hand-side entry point (bp_rhs_noalloc).

It serves callers that cannot allocate device memory -- applications whose
own allocator owns the GPU, or code that must not allocate while another
thread captures a CUDA graph.  Its per-point scratch is a fixed array inside
the library; everything else is caller-owned device memory.  The check:
two calls in a row through the C ABI give the same right-hand side as the
allocating entry point bp_rhs on the same inputs.  Collected last so that a
run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200 import _native as N
from conftest import make_beep, rel_l2

pytestmark = pytest.mark.gpu


def test_rhs_noalloc_matches_bp_rhs():
    import torch
    V, T = b.icosphere(3, 10.0)
    mesh = b.Mesh(V, T, b.charges_in_sphere(10, 7.0, seed=77))
    bp = make_beep(mesh, kappa=0.1)
    ref = bp.set_rhs()  # allocating entry point (bp_rhs)
    g = bp.gathered()
    n = len(g["area"])
    qual = g["qual"]
    nq = len(qual)
    dev = torch.device("cuda", 0)
    off_d = torch.from_numpy(np.ascontiguousarray(g["qual_off"], np.int32)).to(dev)
    soa_d = torch.from_numpy(np.ascontiguousarray(qual.T.reshape(-1))).to(dev)  # 7 arrays of nq doubles
    ch = bp.instances[0].charges
    ch = np.ascontiguousarray(ch[ch[:, 3] != 0])
    ch_d = torch.from_numpy(ch).to(dev)
    out_d = torch.full((2 * n,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream()
    L = N.lib()
    for _ in range(2):  # two calls in a row share the fixed scratch
        out_d.fill_(float("nan"))
        N.check(L.bp_rhs_noalloc(n, off_d.data_ptr(), soa_d.data_ptr(), nq, ch_d.data_ptr(), len(ch), 80.0,
                                 out_d.data_ptr(), C.c_void_p(stream.cuda_stream)))
        stream.synchronize()
        got = out_d.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_l2(got, ref) < 1e-12
    # sizes beyond the fixed scratch are rejected before any launch
    assert L.bp_rhs_noalloc(n, off_d.data_ptr(), soa_d.data_ptr(), (1 << 20) + 1, ch_d.data_ptr(), len(ch), 80.0,
                            out_d.data_ptr(), None) == N.BP_ERR_INVALID
    assert b"exceed the fixed scratch" in L.bp_last_error()
    bp.close()
