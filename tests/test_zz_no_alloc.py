"""kofm_reduce_field_noalloc: the reduction for callers that cannot let the
library allocate device memory (an application serving every device buffer
from its own pool, or a latency-critical caller that cannot take an
allocation's implicit synchronisation).  The caller owns the input field and
the one-double output; the library's only scratch is a fixed 32 KiB array.

Checked through the C ABI against the context-based kofm_reduce on the same
field, on two calls in a row (the shared scratch keeps the previous call's
partials, so the second call must not depend on them).  Runs last so a
failure here leaves every other test already run; it needs no earlier test.
"""
import ctypes as C

import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G


def test_rejects_sizes_beyond_the_scratch_limit(kofm_lib):
    # host-side validation; no device work is queued
    big_rows = _abi.NOALLOC_MAX_NODES // 1024 + 1
    st = kofm_lib.kofm_reduce_field_noalloc(C.c_void_p(16), 1024, 1024, big_rows,
                                            _abi.OP_SUM, C.c_void_p(16), None)
    assert st == _abi.ERR_TOO_LARGE
    assert kofm_lib.kofm_reduce_field_noalloc(None, 8, 8, 8, _abi.OP_SUM, C.c_void_p(16), None) == -200


@pytest.mark.gpu
def test_matches_kofm_reduce_on_two_calls_in_a_row(kofm_lib):
    import torch

    nx, ny = 256, 66
    ch = G.straight_channel(nx, ny)
    d = desc_default()
    d.nx, d.nx_full, d.ny, d.use_komega = nx, nx, ny, 1
    d.tau, d.fterm, d.mu = 1.9, 1e-6, 5e-4
    rng = np.random.default_rng(7)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    with Lattice(d) as L:
        L.set_geometry(ch.ntype, ch.wallD, ch.dX)
        for call in range(2):
            k = rng.uniform(1e-6, 1e-3, ch.n) * ch.fluid_mask().ravel()
            o = rng.uniform(1e-2, 1e1, ch.n) * ch.fluid_mask().ravel()
            L.set_state(G.equilibrium_state(ch), k, o, k / np.maximum(o, 1e-30), np.zeros(3 * ch.n))
            # the caller's own copy of the field in device memory (rows of nx floats)
            kd = torch.from_numpy(k.astype(np.float32)).cuda()
            for op in (_abi.OP_SUM, _abi.OP_MIN, _abi.OP_MAX):
                ref = L.reduce(_abi.FIELD_K, op)
                st = kofm_lib.kofm_reduce_field_noalloc(
                    C.c_void_p(kd.data_ptr()), nx, nx, ny, op, C.c_void_p(out.data_ptr()),
                    C.c_void_p(stream))
                assert st == 0
                torch.cuda.synchronize()
                got = float(out.item())
                if op == _abi.OP_SUM:
                    assert got == pytest.approx(ref, rel=1e-12)
                else:
                    assert got == ref


def _numpy_reduce(a, op):
    return {_abi.OP_SUM: np.sum, _abi.OP_MIN: np.min, _abi.OP_MAX: np.max}[op](a.astype(np.float64))


@pytest.mark.gpu
def test_padded_rows_and_fields_of_several_chunks(kofm_lib):
    """Rows with padding columns (ncols 200 in a pitch of 256, the padding
    filled with +-1e30 so that counting it would show in every operation),
    and a first field of 1024 x 200 nodes -- four 65,536-node chunks, so
    several partials and the final combine's per-thread ranges are used --
    followed by a smaller one (one chunk): the second call reads only the
    partials it wrote itself."""
    import torch

    rng = np.random.default_rng(11)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for (ncols, pitch, ny) in ((200, 256, 1024), (200, 256, 66)):
        a = rng.uniform(-2.0, 3.0, (ny, pitch)).astype(np.float32)
        a[:, ncols:] = np.where(rng.random((ny, pitch - ncols)) < 0.5, 1e30, -1e30)
        ad = torch.from_numpy(a.ravel()).cuda()
        for op in (_abi.OP_SUM, _abi.OP_MIN, _abi.OP_MAX):
            st = kofm_lib.kofm_reduce_field_noalloc(
                C.c_void_p(ad.data_ptr()), ncols, pitch, ny, op, C.c_void_p(out.data_ptr()),
                C.c_void_p(stream))
            assert st == 0
            torch.cuda.synchronize()
            got = float(out.item())
            ref = _numpy_reduce(a[:, :ncols], op)
            if op == _abi.OP_SUM:
                assert got == pytest.approx(ref, rel=1e-12, abs=1e-9)
            else:
                assert got == ref
