"""The Node-side integration sources (integration/node/) against the C ABI.

There is no Node.js here, so the N-API module and the backend object cannot
run.  These checks catch what drifts when the C header changes:
  - binding_b200.cpp type-checks against include/fdtd_b200.h (g++
    -fsyntax-only with a stand-in napi.h that declares the Napi API it uses);
  - every fdtd_* entry point the binding calls is declared in the header and
    exported by libfdtd_b200.so;
  - every addon.<fn> that b200Backend.js calls is registered by the module;
  - b200Backend.js's coefficient and far-field orders are the ones the C
    entry points number (scenario.COEFF_ORDER, scenario.FF_NAMES);
  - registry.patch adds the backend to LOADERS and to the head of the
    selection order (registry.js:13-17,47-50).
"""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT, load_package

pkg = load_package()
from special_topics_b200 import _native as N  # noqa: E402
from special_topics_b200.scenario import COEFF_ORDER, FF_NAMES  # noqa: E402

NODE = os.path.join(ROOT, "integration", "node")


def _read(name):
    with open(os.path.join(NODE, name)) as f:
        return f.read()


def _header_functions():
    src = open(os.path.join(ROOT, "include", "fdtd_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"\b(fdtd_\w+)\s*\(", src))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_binding_type_checks_against_the_header():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror",
                        "-I", os.path.join(ROOT, "tests", "napi_stub"), "-I", os.path.join(ROOT, "include"),
                        os.path.join(NODE, "binding_b200.cpp")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_binding_calls_only_declared_and_exported_entry_points():
    src = re.sub(r"//.*", "", _read("binding_b200.cpp"))
    called = set(re.findall(r"\b(fdtd_\w+)\s*\(", src))
    assert len(called) >= 25
    declared = _header_functions()
    assert called <= declared, sorted(called - declared)
    L = N.lib()
    for name in sorted(called):
        assert hasattr(L, name), name


def test_backend_calls_only_registered_module_functions():
    registered = set(re.findall(r'e\.Set\("(\w+)"', _read("binding_b200.cpp")))
    used = set(re.findall(r"\baddon\.(\w+)\s*\(", _read("b200Backend.js")))
    assert used, "no addon calls found"
    assert used <= registered, sorted(used - registered)


def test_backend_orders_match_the_c_numbering():
    js = _read("b200Backend.js")

    def js_list(name):
        m = re.search(r"\b" + name + r"\s*=\s*\[(.*?)\];", js, flags=re.S)
        return re.findall(r"'(\w+)'", m.group(1))

    assert js_list("COEFF_ORDER") == list(COEFF_ORDER)
    assert js_list("FF_ORDER") == list(FF_NAMES)


def test_registry_patch_registers_b200_first():
    patch = _read("registry.patch")
    added = [ln[1:] for ln in patch.splitlines() if ln.startswith("+") and not ln.startswith("+++")]
    assert any(re.search(r"'b200':\s*\(\)\s*=>\s*import\('\./b200/b200Backend\.js'\)", ln) for ln in added)
    assert any(re.search(r":\s*\['b200', 'webgpu', 'cuda', 'wasm-cpu'\]", ln) for ln in added)
