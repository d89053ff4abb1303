# SPDX-License-Identifier: MIT
"""The C-ABI library loads, exports every symbol include/pmb200_core.h
declares, rejects bad arguments, and fails loudly (no CPU fallback) when no
CUDA device is present."""
import ctypes
import os
import re

import numpy as np
import pytest

from pmb200 import core, scenes

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pmb200_core.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"PMB_API\s+[\w\s\*]+?\b(pmb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(core.LIB_PATH)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_arguments_are_rejected():
    lib = core.lib()
    assert lib.pmb_world_create(None, None) == -1
    assert lib.pmb_world_step(None, None, None) == -1
    assert lib.pmb_world_get_states(None, None) == -1


def test_no_cpu_fallback_without_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(core.PmbError, match="no CUDA device"):
        core.World(scenes.pyramid(levels=2))
    with pytest.raises(core.PmbError, match="no CUDA device"):
        core.math_eval(1, np.zeros((1, 7), np.float32))
