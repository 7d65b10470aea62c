"""Build target in place of the reference's setup_24matching.py
(TR-source/setup_24matching.py:5-33: matching_utils, matching_utils_hash,
matching_utils_bucket, matching_utils_online).  ``python setup_24matching.py
install`` compiles libtrspmm.so and installs the four drop-in modules with
the trspmm package they call."""
import os
import sys

from setuptools import setup

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _setup_common import HERE, package_args  # noqa: E402

setup(name="Matching24", version="2.0",
      py_modules=["matching_utils", "matching_utils_hash", "matching_utils_bucket",
                  "matching_utils_online", "_matching_common"], **package_args())
