"""spring_linewidth3_tetra_noalloc against spring_linewidth3 (tetrahedron), through the C ABI.

The no-alloc entry point serves callers that must not have the library call
cudaMalloc (device memory owned by another allocator, or no synchronising
allocation allowed mid-pipeline).  Its scratch is a fixed device array inside
the library; the caller passes device buffers for the results.  This file is
collected last on purpose, so that a failure here comes after every other test.
"""
import ctypes as ct

import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import _lib as L
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    cr = S.build("rocksalt2")
    N = 6
    st = D.Setup(cr, (N, N, N), [300.0, 700.0])
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    ctx.prepare3()
    lib = L.load()
    nd, nT = ctx.ndof, ctx.n_temps
    for call, i0 in enumerate((2, 5)):
        # the no-alloc call comes first, straight after spring_prepare3: it reads the pair range of
        # its q0 on the device, so nothing before it needs to have read the pair offsets back
        d_lw = torch.full((nT, nd), float("nan"), dtype=torch.float64, device="cuda")
        d_p3 = torch.full((nd,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.spring_linewidth3_tetra_noalloc(ctx._h, i0, None, ct.c_void_p(d_lw.data_ptr()),
                                                 ct.c_void_p(d_p3.data_ptr()))
        assert rc == 0, lib.spring_last_error(ctx._h)
        ctx.synchronize()
        ref, ref_p3 = ctx.linewidth3(i0, 1, delta="tetra")          # allocating entry point
        got = d_lw.cpu().numpy()
        np.testing.assert_allclose(got, ref[:, 0, :], rtol=1e-9, atol=1e-14 * np.abs(ref).max())
        np.testing.assert_allclose(d_p3.cpu().numpy(), ref_p3[0], rtol=1e-9, atol=1e-14 * np.abs(ref_p3).max())
    # a mesh beyond the fixed scratch is refused cleanly
    big = from_crystal(cr, (24, 24, 24), [300.0], phonons="device")[0]
    big.prepare3()
    d_lw = torch.zeros((1, nd), dtype=torch.float64, device="cuda")
    d_p3 = torch.zeros((nd,), dtype=torch.float64, device="cuda")
    rc = lib.spring_linewidth3_tetra_noalloc(big._h, 1, None, ct.c_void_p(d_lw.data_ptr()),
                                             ct.c_void_p(d_p3.data_ptr()))
    assert rc == L.SPRING_ERR_UNSUPPORTED
    big.close()
    ctx.close()
