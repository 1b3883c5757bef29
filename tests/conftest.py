"""Shared pytest configuration: the ``gpu`` marker and common fixtures.

Tests marked ``gpu`` call the CUDA library through its C ABI and need a B200; they fail
(never skip) when no CUDA device is present. Everything else runs on the CPU.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle.load()
