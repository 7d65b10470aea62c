"""Shared part of setup_online.py and setup_24matching.py: the build step
(``make -C csrc``, which compiles libtrspmm.so for sm_100a, a no-op when it
is up to date) run before the Python modules are collected."""
from __future__ import annotations

import os
import subprocess

from setuptools.command.build_py import build_py

HERE = os.path.dirname(os.path.abspath(__file__))


class BuildLibrary(build_py):
    """build_py that first brings trspmm/libtrspmm.so up to date."""

    def run(self):
        subprocess.check_call(["make", "-C", os.path.join(HERE, "csrc")])
        super().run()


def package_args():
    """The trspmm package (with its shared library) every drop-in module imports."""
    return dict(packages=["trspmm", "tr_csr_fp16"], package_dir={"": HERE},
                package_data={"trspmm": ["libtrspmm.so"]}, cmdclass={"build_py": BuildLibrary})
