"""Build target in place of the reference's setup_online.py scripts
(TR-source/setup_online.py:5-18 builds Libra5BlockOnline, the router;
TR-source/SpMM/setup_online.py:5-22 builds Libra6SpMMOnline, the
operators).  ``python setup_online.py install`` (or ``build_ext
--inplace``-style ``build_py``) compiles libtrspmm.so and installs both
drop-in modules with the trspmm package they call, so
``import Libra5BlockOnline`` / ``import Libra6SpMMOnline`` work as after
the reference's build."""
import os
import sys

from setuptools import setup

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _setup_common import HERE, package_args  # noqa: E402

setup(name="Libra6Online", version="2.0",
      py_modules=["Libra5BlockOnline", "Libra6SpMMOnline"], **package_args())
