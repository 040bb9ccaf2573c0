"""The compaction entry point that allocates nothing, checked against the step's own list.

`fp_compact_ids_noalloc` serves callers that cannot allocate device memory where they call
it (a frame loop that must not stall on cudaMalloc, a host that owns every device byte, code
inside a stream capture); its scratch is an array inside the library. This test gives it
the flags "brick has a slot" read from a simulation and compares its ascending ids with the
computing-brick list the simulation's allocation produced (FP_TABLE_ACTIVE), exactly, on
two calls in a row over two different steps. The file sorts last so a stop-at-first-failure
run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from firepro import abi, scenes
from firepro.engine import FluidSimulation

pytestmark = pytest.mark.gpu


def test_compact_noalloc_matches_active_list():
    import torch

    lib = abi.load_library()
    sc = scenes.SinglePlume()
    sim = FluidSimulation(sc.grid(budget=2 ** 19))
    sim.set_runtime(0.05, 2 ** 19, True)
    step = 0
    for call in range(2):
        for _ in range(3):
            sim.step(sc.frame(step).frame)
            step += 1
        entries = sim.table(abi.FP_TABLE_ENTRIES).view(np.int32)
        expected = sim.table(abi.FP_TABLE_ACTIVE)
        n = entries.size
        flags = torch.from_numpy((entries >= 0).astype(np.int32)).cuda()
        ids = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        count = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = lib.fp_compact_ids_noalloc(C.c_void_p(flags.data_ptr()), n, C.c_void_p(ids.data_ptr()),
                                        C.c_void_p(count.data_ptr()), None)
        assert rc == abi.FP_OK, lib.fp_last_error(None).decode()
        torch.cuda.synchronize()
        k = int(count.item())
        assert k == int(expected[0]) and k > 0, (call, k, int(expected[0]))
        assert np.array_equal(ids[:k].cpu().numpy().astype(np.uint32), expected[1:1 + k]), call
    sim.dispose()


def test_compact_noalloc_rejects_oversize():
    lib = abi.load_library()
    rc = lib.fp_compact_ids_noalloc(None, abi.FP_COMPACT_MAX_IDS + 1, None, None, None)
    assert rc == abi.FP_ELIMIT
    assert "exceeds FP_COMPACT_MAX_IDS" in lib.fp_last_error(None).decode()
