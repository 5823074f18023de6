"""The C-ABI library loads and exports every function include/*.h declares.
No compute call is made (no GPU needed)."""
import ctypes
import glob
import os
import re

from aviatorengine2_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(ae_\w+)\s*\(", src):
            if not re.search(r"typedef[^;]*\b" + m.group(1) + r"\b", src):
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    names = declared_functions()
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_error_paths_without_device():
    L = _lib.lib()
    # Null contexts are rejected before any CUDA call.
    assert L.ae_set_config(None, None) == -1
    assert L.ae_closest_hit(None, None, 0, None, 0) == -1
    assert L.ae_render_frame(None, 0, None) == -1
    assert L.ae_last_error(None) == b"null context"
