"""Loader of the reference's own CUDA extension rebuilt for sm_100a
(``make -C oracle ref`` -> oracle/_ref).  Test infrastructure: the reference
module is a checker only."""

from __future__ import annotations

import importlib.machinery
import importlib.util
import sysconfig
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
REF_SO = ROOT / "oracle" / "_ref" / f"_cuda_backend{sysconfig.get_config_var('EXT_SUFFIX')}"


def load_reference_module():
    """The reference's ``standalone_backend._cuda_backend`` (under the plain
    name ``_cuda_backend``), or None when oracle/_ref was not built."""
    if not REF_SO.exists():
        return None
    loader = importlib.machinery.ExtensionFileLoader("_cuda_backend", str(REF_SO))
    spec = importlib.util.spec_from_loader("_cuda_backend", loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod
