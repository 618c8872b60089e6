"""gva_step_run_static: the step launcher for callers that cannot allocate
device memory at call time (its scratch is a fixed array in the library).

Checked through the C ABI against gva_step_run (caller-provided scratch) on
the same inputs, over every step of a plan, for two complete passes in a row:
the shared array keeps the previous call's contents, and the results must not
depend on them.  Integer rows: compared bit for bit.  Collected last (zz) so
that a failure here leaves every other test already run; passes alone too.
"""
import ctypes

import numpy as np
import pytest

import geneva_b200 as gv
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

QUERY = "v 0 1\nv 1 1\nv 2 2\nv 3 3\ne 0 1 1\ne 1 2 1\ne 2 3 2\ne 0 2 2\n"


def _declare(lib):
    vp, u64 = ctypes.c_void_p, ctypes.c_uint64
    lib.gva_step_run_static.restype = ctypes.c_int
    lib.gva_step_run_static.argtypes = [vp, vp, ctypes.c_int, vp, u64, vp, u64, ctypes.POINTER(u64), vp]
    return lib


def _chain(lib, torch, db, plan, static: bool):
    """Runs every step, growing the output to the reported size when needed."""
    stream = torch.cuda.current_stream().cuda_stream
    cur, rows, outs = None, 0, []
    for s in range(lib.gva_plan_num_steps(plan._h, db._h)):
        wout = lib.gva_plan_step_width_out(plan._h, db._h, s)
        n = ctypes.c_uint64()
        cap = max(1, 4 * rows + 1024)
        for _ in range(2):
            out = torch.empty(cap * wout, dtype=torch.int32, device="cuda")
            inp = cur.data_ptr() if cur is not None else None
            if static:
                st = lib.gva_step_run_static(db._h, plan._h, s, inp, rows, out.data_ptr(), cap, ctypes.byref(n),
                                             stream)
            else:
                scratch = torch.empty(max(1, lib.gva_step_scratch_bytes(rows)), dtype=torch.uint8, device="cuda")
                st = lib.gva_step_run(db._h, plan._h, s, inp, rows, out.data_ptr(), cap, ctypes.byref(n),
                                      scratch.data_ptr(), scratch.numel(), stream)
            if st != 4:  # 4 = capacity too small; n holds the needed rows
                break
            cap = n.value
        assert st == 0, lib.gva_last_error()
        rows = n.value
        cur = out[: rows * wout]
        torch.cuda.synchronize()
        outs.append(cur.cpu().numpy().view(np.uint32).reshape(rows, wout).copy())
    return outs


def test_static_scratch_matches_caller_scratch(native):
    torch = pytest.importorskip("torch")
    lib = _declare(native)
    g = GOLDEN / "graphs"
    db = gv.loadDataBase(g / "syn_hub.mygraph", g / "syn_hub.metadata")
    plan = gv.Plan.from_text(QUERY)
    want = _chain(lib, torch, db, plan, static=False)
    assert want[-1].shape[0] > 0
    first = _chain(lib, torch, db, plan, static=True)   # sets up the array on this device
    second = _chain(lib, torch, db, plan, static=True)  # reuses it with the previous contents
    assert len(want) == len(first) == len(second)
    for w, a, b in zip(want, first, second):
        assert np.array_equal(w, a)
        assert np.array_equal(w, b)
    db.close()


def test_static_scratch_rejects_oversized_input(native):
    lib = _declare(native)
    g = GOLDEN / "graphs"
    db = gv.loadDataBase(g / "syn_a.mygraph", g / "syn_a.metadata")
    plan = gv.Plan.from_text(QUERY)
    n = ctypes.c_uint64()
    # the size is checked on the host before anything is launched
    st = lib.gva_step_run_static(db._h, plan._h, 1, None, (1 << 24) + 1, None, 1, ctypes.byref(n), None)
    assert st == 5
    assert b"GVA_STATIC_MAX_ROWS" in lib.gva_last_error()
    db.close()
