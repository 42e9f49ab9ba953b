"""Shared test setup.

``-m gpu`` tests need an sm_100 device and call the CUDA library through its C
ABI; everything else runs on the CPU.  The CPU oracle (oracle/) is built on
first use; the CUDA library must already be built (``python -m
gargantua_b200.build``; ``__graft_entry__.build()`` does both).
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gglib():
    from gargantua_b200 import abi, build
    build.build()
    return abi.load()


@pytest.fixture(scope="session")
def renderer(gglib):
    from gargantua_b200.curved import Renderer
    r = Renderer(0)
    yield r
    r.close()
