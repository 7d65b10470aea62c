"""The build targets that stand in for the reference's setup_online.py and
setup_24matching.py: building them into a fresh directory gives importable
drop-in modules (the library is already built in the tree, so make is a
no-op)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "tr-spmm_b200")


@pytest.mark.parametrize("script, modules", [
    ("setup_online.py", ["Libra5BlockOnline", "Libra6SpMMOnline"]),
    ("setup_24matching.py", ["matching_utils", "matching_utils_hash", "matching_utils_bucket",
                             "matching_utils_online"]),
])
def test_build_target_installs_importable_modules(tmp_path, script, modules):
    out = tmp_path / "lib"
    subprocess.run([sys.executable, script, "-q", "build_py", "--build-lib", str(out)],
                   cwd=PKG, check=True, capture_output=True, timeout=600)
    assert (out / "trspmm" / "libtrspmm.so").is_file()
    code = ("import sys; sys.path.insert(0, %r); " % str(out) +
            "; ".join(f"import {m}" for m in modules) +
            "; import trspmm; assert trspmm.LIB_PATH.startswith(%r)" % str(out))
    env = {k: v for k, v in os.environ.items() if k != "PYTHONPATH"}
    subprocess.run([sys.executable, "-c", code], cwd=str(tmp_path), check=True, env=env,
                   timeout=300)
