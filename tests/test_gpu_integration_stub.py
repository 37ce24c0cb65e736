"""The ctypes binding INTEGRATION.md gives a maintainer of the reference, run
as written there.

The stub is read from INTEGRATION.md itself (the Python block under "Binding
a maintainer would add to the reference") and executed unchanged from the
repository root, so the documented one-call host entry ``pfx_parflex`` is what
is tested: host C in, ``(best_cost, wp)`` out, bit-exact against the
reference's own results on every stage-2 golden fixture, and the reference's
ValueError when no endpoint qualifies (Parflex.py:1285-1286).
"""
import os
import re

import numpy as np
import pytest

from golden_util import load, names

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parflexdtw_b200 import workloads as W  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _stub_source():
    with open(os.path.join(ROOT, "INTEGRATION.md")) as fp:
        text = fp.read()
    sec = text.split("## Binding a maintainer would add to the reference", 1)[1]
    m = re.search(r"```python\n(.*?)```", sec, re.S)
    assert m, "no Python block in the binding section"
    return m.group(1)


@pytest.fixture(scope="module")
def stub():
    cwd = os.getcwd()
    os.chdir(ROOT)  # the stub names the library by its path in the checkout
    try:
        ns = {}
        exec(compile(_stub_source(), "INTEGRATION.md", "exec"), ns)
    finally:
        os.chdir(cwd)
    return ns["parflex"]


@pytest.mark.parametrize("name", names("stage2"))
def test_stub_parflex_golden(stub, name):
    g = load("stage2", name)
    best, wp = stub(g["C"], g["steps"], g["weights"], float(g["beta"]), L=int(g["L"]))
    assert best == float(g["best_cost"])
    assert wp.dtype == np.int64 and np.array_equal(wp, g["wp"])


def test_stub_parflex_no_endpoint(stub):
    rng = np.random.default_rng(3)
    F1, F2 = W.warped_pair(rng, 200, 200)
    C = W.cost_matrix_det(F1, F2)
    with pytest.raises(ValueError, match="No valid endpoint"):
        stub(C, [(1, 1), (1, 2), (2, 1)], [2, 3, 3], 1.0, L=50)
