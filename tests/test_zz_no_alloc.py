"""wql3d_max_abs_noalloc: the reduction for callers that cannot allocate GPU memory.

A Fortran driver that keeps its device data in fixed OpenACC data regions
(and audits that time stepping allocates nothing) still needs the final-state
max|field| diagnostic.  The allocation-free entry point reduces a device array
the caller owns, into outputs the caller owns, with only the library's static
scratch.  This file checks it against the regular entry point
(wql3d_final_state) on two calls in a row; it is collected last so a failure
here never hides another test.
"""
import ctypes as C

import numpy as np
import pytest

from cases import small_case

pytestmark = pytest.mark.gpu


def _noalloc_max(L, t, stream=None):
    import torch
    res = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    flag = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    rc = L.wql3d_max_abs_noalloc(C.c_void_p(t.data_ptr()), t.numel(), C.c_void_p(res.data_ptr()),
                                 C.c_void_p(flag.data_ptr()), stream)
    assert rc == 0, L.wql3d_last_error()
    torch.cuda.synchronize()
    return float(res.item()), int(flag.item())


def test_noalloc_max_matches_final_state_twice(wql3d_lib):
    import torch
    from waveqlab3d_q_gpu_b200.domain import Domain
    L = wql3d_lib
    # call 1: a 21x23x25 block after 6 steps, scaled up so that its partial
    # maxima dominate anything a later, smaller call could read by mistake
    p1 = small_case(n=(21, 23, 25))
    g1 = Domain(p1, nsteps_hint=8)
    g1.run(6)
    ref1, _, _ = g1.final_state()
    F1 = torch.tensor(g1.fields(host_nb=3), device="cuda") * 1000.0
    got1, bad1 = _noalloc_max(L, F1)
    assert got1 == 1000.0 * ref1 and bad1 == 0
    # call 2: a smaller block (fewer scratch slots in use) right after
    p2 = small_case(n=(15, 16, 17), seed=5)
    g2 = Domain(p2, nsteps_hint=8)
    g2.run(4)
    ref2, _, _ = g2.final_state()
    F2 = torch.tensor(g2.fields(host_nb=3), device="cuda")
    got2, bad2 = _noalloc_max(L, F2)
    assert got2 == ref2 and bad2 == 0
    assert got2 < got1
    # non-finite state: flagged like wql3d_final_state's WQL3D_ENONFINITE
    F2[4, 3, 5, 7] = float("nan")
    bad_host = F2[:, 3:-3, 3:-3, 3:-3].cpu().numpy()
    g2.set_fields(bad_host)
    rc = L.wql3d_final_state(g2.handle, None, None, None)
    _, bad3 = _noalloc_max(L, F2)
    assert rc == -4 and bad3 == 1
    g1.close()
    g2.close()


def test_noalloc_second_call_allocates_no_device_memory(wql3d_lib):
    """After the first call on the device (set-up), a call leaves the device's
    free memory unchanged: inputs and outputs are the caller's, the scratch is
    the library's static array."""
    import torch
    L = wql3d_lib
    a = torch.linspace(-3.0, 2.0, 1 << 20, dtype=torch.float64, device="cuda")
    res = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    flag = torch.full((1,), -1, dtype=torch.int32, device="cuda")

    def call():
        rc = L.wql3d_max_abs_noalloc(C.c_void_p(a.data_ptr()), a.numel(), C.c_void_p(res.data_ptr()),
                                     C.c_void_p(flag.data_ptr()), None)
        assert rc == 0, L.wql3d_last_error()
        torch.cuda.synchronize()

    call()
    free0, _ = torch.cuda.mem_get_info()
    call()
    call()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert float(res.item()) == 3.0 and int(flag.item()) == 0


def test_noalloc_rejects_sizes_beyond_the_scratch(wql3d_lib):
    L = wql3d_lib
    limit = 65536 * 8192
    res = C.c_double()
    rc = L.wql3d_max_abs_noalloc(C.c_void_p(1), limit + 1, C.byref(res), None, None)
    assert rc == -1
    assert b"exceeds the fixed scratch limit" in L.wql3d_last_error()
