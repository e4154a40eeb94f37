"""pytest plugin: run the reference's own test files, unchanged, against
this package.

The reference's tests import ``warp`` only for ``wp.is_cuda_available()``
(tests/test_cavity.py:15,62; tests/test_mg.py:7,56) and put the reference
checkout first on ``sys.path`` before importing ``warpflow``.  Loaded with
``-p wf_refsuite_plugin`` (this folder and the package folder on
PYTHONPATH), the plugin imports this package's ``warpflow`` modules first,
so that the reference's imports resolve to them, and installs a one-function
``warp`` module whose ``is_cuda_available()`` is torch's.
"""
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(os.path.dirname(HERE)), "warpflow-les_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

import torch  # noqa: E402

import warpflow  # noqa: E402,F401
import warpflow.config  # noqa: E402,F401
import warpflow.multigrid  # noqa: E402,F401
import warpflow.solver  # noqa: E402,F401
import warpflow.topology  # noqa: E402,F401

_warp = types.ModuleType("warp")
_warp.is_cuda_available = torch.cuda.is_available
sys.modules["warp"] = _warp
