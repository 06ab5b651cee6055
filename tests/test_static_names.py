"""Every global name a function of the Python sources refers to exists --
a NameError in a path that only runs on a GPU (bench.py's GPU arm, the
device helpers of the binding) is otherwise found only there.  Uses the
compiler's own symbol tables; CPU only."""
import builtins
import os
import symtable

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FILES = ["bench.py", "__graft_entry__.py", "gpu-canonical-labeling_b200/api.py",
         "gpu-canonical-labeling_b200/graphs.py", "gpu-canonical-labeling_b200/build.py",
         "gpu-canonical-labeling_b200/__init__.py", "oracle/oracle.py"]
# the tests too: those marked gpu or gpu_staged run only on a GPU
FILES += sorted(os.path.join("tests", f) for f in os.listdir(os.path.join(ROOT, "tests"))
                if f.startswith("test_") and f.endswith(".py"))
FILES += ["tests/conftest.py", "tests/golden/make_golden.py"]


def _module_names(top):
    names = set()
    for sym in top.get_symbols():
        if sym.is_assigned() or sym.is_imported() or sym.is_namespace():
            names.add(sym.get_name())
    return names


def _undefined(table, defined):
    bad = []
    for sym in table.get_symbols():
        name = sym.get_name()
        if (sym.is_global() and not sym.is_declared_global() and sym.is_referenced()
                and name not in defined and not hasattr(builtins, name)):
            bad.append((table.get_name(), table.get_lineno(), name))
    for child in table.get_children():
        bad += _undefined(child, defined)
    return bad


@pytest.mark.parametrize("path", FILES)
def test_global_names_resolve(path):
    src = open(os.path.join(ROOT, path)).read()
    top = symtable.symtable(src, path, "exec")
    defined = _module_names(top) | {"__file__", "__name__", "__doc__", "__spec__",
                                    "__path__", "__package__"}
    assert _undefined(top, defined) == []
