"""CPU checks of the drop-in boundary: the C-ABI library loads, exports every
entry point include/zpic_b200.h declares, and fails loudly without a GPU."""
import os
import re
import subprocess

import pytest

import zpic_b200 as zb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'zpic_b200.h')


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r'\b(zpic_b200_\w+)\s*\(', src)))


def test_header_lists_match_binding():
    assert declared() == sorted(zb.EXPORTS)


def test_library_exports_every_symbol():
    lib = zb.lib()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.check_output(['nm', '-D', '--defined-only', zb.LIB_PATH]).decode()
    exported = set(re.findall(r' T (zpic_b200_\w+)', out))
    assert set(declared()) <= exported


def test_version_and_error_channel():
    assert zb.lib().zpic_b200_version() >= 10000
    assert isinstance(zb.lib().zpic_b200_last_error(), bytes)


def test_courant_violation_rejected():
    # EMF ctor (emf.cpp:20-28): dt >= Courant limit is an error, reported before any device work
    with pytest.raises(zb.ZpicError, match='courant'):
        zb.Simulation((2, 2), (16, 16), (3.2, 3.2), 0.5)


def test_invalid_tiles_rejected():
    with pytest.raises(zb.ZpicError, match='tiles'):
        zb.Simulation((0, 2), (16, 16), (3.2, 3.2), 0.05)


def test_no_silent_cpu_fallback():
    """Without a CUDA device creating a simulation raises; nothing runs on the CPU instead."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    with pytest.raises(zb.ZpicError):
        zb.Simulation((2, 2), (16, 16), (3.2, 3.2), 0.05)
