"""cup2d_adv_diff_noalloc: the allocation-free advDiff entry point.

Callers that cannot allocate device memory (their own pool owns the GPU's
memory, or their loop must not pay cudaMalloc's device synchronisation) get
advDiff on buffers they own, with the reduction scratch held in a fixed
array inside the library.  This test calls it through the C ABI twice in a
row on the same inputs and checks both results against the context-based
entry point cup2d_adv_diff, within the advDiff tolerance of the parity tests
(1e-14 relative: only the boundary outflow sum is a reduction).  It lives in
a file pytest collects last and needs nothing from the other test files.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ARGS = ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace "
        "-shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_adv_diff_noalloc_matches_context_entry_point_twice():
    import torch
    from cubismup_2d_b200 import Simulation, abi
    from cubismup_2d_b200.synthetic import noise_field

    sim = Simulation(ARGS)
    sim.init()
    ctx = sim.ctx
    u0 = ctx.get("u") + noise_field(21, 0, ctx.ny, ctx.nx, amp=1e-2)
    v0 = ctx.get("v") + noise_field(21, 1, ctx.ny, ctx.nx, amp=1e-2)
    ctx.set("u", u0)
    ctx.set("v", v0)
    st = ctx.scalars()
    dt = 1e-3
    ctx.adv_diff(dt)
    ref_u, ref_v = ctx.get("u"), ctx.get("v")

    dev = torch.device("cuda", 0)
    du = torch.from_numpy(u0).to(dev)
    dv = torch.from_numpy(v0).to(dev)
    L = abi.lib()
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        ou = torch.full_like(du, float("nan"))
        ov = torch.full_like(dv, float("nan"))
        torch.cuda.synchronize()
        rc = L.cup2d_adv_diff_noalloc(
            ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(dv.data_ptr()),
            ctypes.c_void_p(ou.data_ptr()), ctypes.c_void_p(ov.data_ptr()),
            sim.cfg.bpdx, sim.cfg.bpdy, ctx.h, sim.cfg.nu, dt, st["uinfx"], st["uinfy"],
            ctypes.c_void_p(stream.cuda_stream))
        assert rc == abi.OK, (call, rc)
        torch.cuda.synchronize()
        assert rel_err(ou.cpu().numpy(), ref_u) <= 1e-14, call
        assert rel_err(ov.cpu().numpy(), ref_v) <= 1e-14, call


def test_adv_diff_noalloc_rejects_grids_beyond_its_scratch():
    from cubismup_2d_b200 import abi
    L = abi.lib()
    # checked before any device access: the pointers are never dereferenced
    one = ctypes.c_void_p(256)
    rc = L.cup2d_adv_diff_noalloc(one, one, ctypes.c_void_p(512), ctypes.c_void_p(768),
                                  256, 128, 1e-3, 1e-3, 1e-4, 0.0, 0.0, None)
    assert rc == abi.ETOOLARGE
