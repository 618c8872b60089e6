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


def test_static_scratch_accepts_the_maximum_input(native):
    """Exactly GVA_STATIC_MAX_ROWS input rows fit the fixed array: the step runs
    (count pass over every row) and reports the rows it would write instead of
    an argument error."""
    torch = pytest.importorskip("torch")
    lib = _declare(native)
    g = GOLDEN / "graphs"
    db = gv.loadDataBase(g / "syn_hub.mygraph", g / "syn_hub.metadata")
    plan = gv.Plan.from_text(QUERY)
    assert lib.gva_plan_step_width_in(plan._h, db._h, 1) == 1
    max_rows = 1 << 24
    # the seed step's vertices repeated up to the maximum row count
    n0 = ctypes.c_uint64()
    seed = torch.empty(1 << 16, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.gva_step_run_static(db._h, plan._h, 0, None, 0, seed.data_ptr(), seed.numel(), ctypes.byref(n0), stream)
    assert st == 0 and n0.value > 0, lib.gva_last_error()
    base = seed[: n0.value]
    inp = base.repeat((max_rows + n0.value - 1) // n0.value)[:max_rows].contiguous()
    torch.cuda.synchronize()
    n = ctypes.c_uint64()
    st = lib.gva_step_run_static(db._h, plan._h, 1, inp.data_ptr(), max_rows, None, 0, ctypes.byref(n), stream)
    # the same step on one copy of the seed rows, caller scratch
    n1 = ctypes.c_uint64()
    scratch = torch.empty(lib.gva_step_scratch_bytes(n0.value), dtype=torch.uint8, device="cuda")
    st1 = lib.gva_step_run(db._h, plan._h, 1, base.data_ptr(), n0.value, None, 0, ctypes.byref(n1),
                           scratch.data_ptr(), scratch.numel(), stream)
    assert st1 in (0, 4), lib.gva_last_error()
    assert st in (0, 4), lib.gva_last_error()  # 4: the output does not fit (capacity 0); never an argument error
    reps, rest = divmod(max_rows, n0.value)
    n_rest = ctypes.c_uint64()
    if rest:
        st2 = lib.gva_step_run(db._h, plan._h, 1, base.data_ptr(), rest, None, 0, ctypes.byref(n_rest),
                               scratch.data_ptr(), scratch.numel(), stream)
        assert st2 in (0, 4), lib.gva_last_error()
    assert n.value == reps * n1.value + n_rest.value
    db.close()
