"""Host-side checks of the pipelined I/O bindings (FlowFieldSet.io_*): the
buffers a caller hands over are validated before any pointer reaches the C
ABI (float64, contiguous, exactly one block's prim), for numpy arrays and
torch tensors alike.  No GPU: the check runs before the library call."""
import numpy as np
import pytest
import torch

from orion_b200 import cases, solver
from orion_b200._lib import OrionError


def _bare_case():
    fs = object.__new__(solver.FlowFieldSet)  # no device case: only the layout is read
    fs.case = cases.small_case(name="io_cpu", dims=(25, 17, 13), split=(2, 1, 1))
    return fs


def test_prim_buffers_of_the_right_layout_pass():
    fs = _bare_case()
    for b, blk in enumerate(fs.case.blocks):
        n = 6 * int(np.prod(blk.padded))
        a = np.zeros(n)
        assert fs._prim_buffer(b, a) == a.ctypes.data
        t = torch.zeros(n, dtype=torch.float64)
        assert fs._prim_buffer(b, t) == t.data_ptr()


@pytest.mark.parametrize("bad", ["float32", "short", "strided"])
def test_prim_buffers_of_another_layout_are_refused(bad):
    fs = _bare_case()
    n = 6 * int(np.prod(fs.case.blocks[0].padded))
    if bad == "float32":
        arrs = [np.zeros(n, dtype=np.float32), torch.zeros(n, dtype=torch.float32)]
    elif bad == "short":
        arrs = [np.zeros(n - 1), torch.zeros(n - 1, dtype=torch.float64)]
    else:
        arrs = [np.zeros(2 * n)[::2], torch.zeros(2 * n, dtype=torch.float64)[::2]]
    for a in arrs:
        with pytest.raises(OrionError):
            fs._prim_buffer(0, a)
