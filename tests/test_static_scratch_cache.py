"""CPU check of the per-(device, context) address cache behind
gb_forward_static_scratch: a call on a context not seen before looks the
static array's address up again instead of reusing another context's
(tests/symcache_check.cpp, built with the host C++ compiler)."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_symbol_cache_relooks_up_on_a_new_context():
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.fail("no C++ compiler on PATH")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "symcache_check")
        subprocess.run([cxx, "-std=c++17", "-O1", "-pthread", "-o", exe, os.path.join(HERE, "symcache_check.cpp")],
                       check=True)
        r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
