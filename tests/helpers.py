"""Shared test helpers: load the package (its directory name is not an
identifier) and the oracle, and build both libraries when missing."""
from __future__ import annotations

import importlib.util
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "gpu-path-delay-coverage_b200"


def _load(name: str, path: Path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def ensure_built() -> None:
    if not (PKG_DIR / "libpdf_b200.so").exists():
        subprocess.run(["make", "-s", "-j4", "-C", str(PKG_DIR)], check=True)
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)


def pdf():
    ensure_built()
    return _load("pdf_b200", PKG_DIR / "__init__.py")


def oracle():
    ensure_built()
    return _load("pdf_oracle", ROOT / "oracle" / "oracle.py")


def rand_codes(rng: np.random.Generator, rows: int, n: int) -> np.ndarray:
    return rng.integers(0, 4, size=(rows, n), dtype=np.uint8)
