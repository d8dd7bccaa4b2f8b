"""CPU checks of the C ABI: the library loads without a GPU, exports every entry point that
include/cy3q.h declares, and refuses to compute without a device (no CPU fallback)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    inc = os.path.join(ROOT, "include")
    src = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cy3q_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def L():
    from papers_b200 import build as b

    b.build()
    from papers_b200 import cy3q

    return cy3q.lib()


def test_library_exports_every_declared_symbol(L):
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []


def test_python_binding_covers_header(L):
    from papers_b200 import cy3q, ty

    assert sorted(cy3q.EXPORTS + ty.TY_EXPORTS) == _declared()


def test_no_cpu_fallback_without_gpu(L):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from papers_b200 import Cy3qError, QuinticSolver

    with pytest.raises(Cy3qError) as e:
        QuinticSolver(3, 100, 1)
    assert "no CUDA device" in str(e.value)


def test_product_package_does_not_import_oracle():
    pkg = os.path.join(ROOT, "papers_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                txt = open(os.path.join(dirpath, f), errors="replace").read()
                assert "import oracle" not in txt and "liboracle" not in txt, f
