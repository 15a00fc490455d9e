"""Build recipe for the reference's own ``src/bem`` CUDA extension (test oracle only).

This is test infrastructure.  It compiles the reference's unmodified
``src/bem/cuda/bind.cu`` (plus its ``include/`` headers) exactly where the
sources lie under the read-only reference checkout, with our own build
directory ``oracle/_ref/`` (git-ignored, but shipped with the tree so the
prebuilt ``.so`` can be imported on a machine without the reference sources).

The reference's own loader (``src/bem/solver.py:9-31``) forces
``TORCH_EXTENSIONS_DIR`` into the source tree and builds at import time; we do
not run it.  We pass the same nvcc flags it passes for a release build
(``--extended-lambda --expt-relaxed-constexpr -O3 -DNDEBUG``,
``src/bem/solver.py:12-18``) and target Blackwell (sm_100).

Only ``tests/`` and the golden-fixture generator may import the result, via
:func:`load_prebuilt`.
"""
from __future__ import annotations

import importlib.machinery
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
MODULE_NAME = "neuralat_ref_bem"
# The reference checkout: $NEURALAT_REFERENCE, else a directory named
# "reference" beside this repository.
DEFAULT_REFERENCE = os.environ.get(
    "NEURALAT_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def so_path() -> str:
    return os.path.join(REF_DIR, MODULE_NAME + ".so")


def build(reference_root: str = DEFAULT_REFERENCE, verbose: bool = False) -> str | None:
    """Compile the reference extension into ``oracle/_ref``; return the .so path.

    Returns None when the reference checkout is absent (e.g. on a GPU box that
    only received the prebuilt files).
    """
    src_dir = os.path.join(reference_root, "src", "bem", "cuda")
    bind = os.path.join(src_dir, "bind.cu")
    if not os.path.exists(bind):
        return None
    out = so_path()
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(bind):
        return out
    os.makedirs(REF_DIR, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    from torch.utils.cpp_extension import load

    load(
        name=MODULE_NAME,
        sources=[bind],
        extra_include_paths=[os.path.join(src_dir, "include")],
        extra_cuda_cflags=["--extended-lambda", "--expt-relaxed-constexpr", "-O3", "-DNDEBUG"],
        build_directory=REF_DIR,
        verbose=verbose,
        is_python_module=True,
    )
    return out


def load_prebuilt():
    """Import the prebuilt reference extension (requires ``import torch`` first)."""
    import torch  # noqa: F401  (loads libtorch / libc10 the extension links against)

    path = so_path()
    if not os.path.exists(path):
        return None
    if MODULE_NAME in sys.modules:
        return sys.modules[MODULE_NAME]
    loader = importlib.machinery.ExtensionFileLoader(MODULE_NAME, path)
    spec = importlib.util.spec_from_file_location(MODULE_NAME, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    sys.modules[MODULE_NAME] = mod
    return mod


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_REFERENCE, verbose=True))
