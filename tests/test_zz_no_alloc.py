"""cup2d_adv_diff_noalloc: the allocation-free advDiff entry point.

Callers that cannot allocate device memory (their own pool owns the GPU's
memory, or their loop must not pay cudaMalloc's device synchronisation) get
advDiff on buffers they own, with the reduction scratch held in a fixed
array inside the library.  This test calls it through the C ABI twice in a
row on one stream (the second call advances the first's result) and checks
both results against the context-based entry point cup2d_adv_diff, within
the advDiff tolerance of the parity tests (1e-14 relative: only the
boundary outflow sum is a reduction).  It lives in a file pytest collects
last and needs nothing from the other test files.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def args_for(bpdx, bpdy):
    """A forced disk in the middle of a bpdx x bpdy block grid of extent 1."""
    h = 1.0 / (32 * max(bpdx, bpdy))
    X, Y = 32 * bpdx * h, 32 * bpdy * h
    R = 0.2 * min(X, Y)
    return (f"-bpdx {bpdx} -bpdy {bpdy} -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace "
            f"-shapes 'disk radius={R} xpos={X / 2} ypos={Y / 2} bForced=1 bFixed=1 xvel=0.2'")


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# one block (every boundary of the grid in one CTA), a row of blocks, the
# small square-ish grid and a 2048 x 1024 grid
@pytest.mark.parametrize("bpdx,bpdy", [(1, 1), (3, 1), (4, 2), (64, 32)])
def test_adv_diff_noalloc_matches_context_entry_point_twice(bpdx, bpdy):
    """Two calls in a row on one stream, with no synchronisation between
    them (the second reads the first's output), each checked against
    cup2d_adv_diff applied to the same state."""
    import torch
    from cubismup_2d_b200 import Simulation, abi
    from cubismup_2d_b200.synthetic import noise_field

    sim = Simulation(args_for(bpdx, bpdy))
    sim.init()
    ctx = sim.ctx
    u0 = ctx.get("u") + noise_field(21, 0, ctx.ny, ctx.nx, amp=1e-2)
    v0 = ctx.get("v") + noise_field(21, 1, ctx.ny, ctx.nx, amp=1e-2)
    st = ctx.scalars()
    dt = 1e-3
    # the reference results of both calls: advDiff of the start state, then
    # advDiff of that result
    refs = []
    ctx.set("u", u0)
    ctx.set("v", v0)
    for call in range(2):
        ctx.adv_diff(dt)
        refs.append((ctx.get("u"), ctx.get("v")))
        ctx.set("u", refs[-1][0])                 # back into step order
        ctx.set("v", refs[-1][1])

    dev = torch.device("cuda", 0)
    bufs = [(torch.from_numpy(u0).to(dev), torch.from_numpy(v0).to(dev))]
    for call in range(2):
        bufs.append((torch.full_like(bufs[0][0], float("nan")), torch.full_like(bufs[0][1], float("nan"))))
    L = abi.lib()
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    for call in range(2):
        (iu, iv), (ou, ov) = bufs[call], bufs[call + 1]
        rc = L.cup2d_adv_diff_noalloc(
            ctypes.c_void_p(iu.data_ptr()), ctypes.c_void_p(iv.data_ptr()),
            ctypes.c_void_p(ou.data_ptr()), ctypes.c_void_p(ov.data_ptr()),
            bpdx, bpdy, ctx.h, sim.cfg.nu, dt, st["uinfx"], st["uinfy"],
            ctypes.c_void_p(stream.cuda_stream))
        assert rc == abi.OK, (call, rc)
    torch.cuda.synchronize()
    for call in range(2):
        ou, ov = bufs[call + 1]
        assert rel_err(ou.cpu().numpy(), refs[call][0]) <= 1e-14, call
        assert rel_err(ov.cpu().numpy(), refs[call][1]) <= 1e-14, call


def test_adv_diff_noalloc_rejects_grids_beyond_its_scratch():
    from cubismup_2d_b200 import abi
    L = abi.lib()
    # checked before any device access: the pointers are never dereferenced
    one = ctypes.c_void_p(256)
    rc = L.cup2d_adv_diff_noalloc(one, one, ctypes.c_void_p(512), ctypes.c_void_p(768),
                                  256, 128, 1e-3, 1e-3, 1e-4, 0.0, 0.0, None)
    assert rc == abi.ETOOLARGE
