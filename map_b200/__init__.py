"""B200-native map-algebra engine.

The user-facing module is `map_b200.map` (also importable as plain `map` with
this directory on sys.path, which is how scripts written for the reference's
Python bindings run unchanged). The native library is map_b200/libmap_b200.so,
built in-tree by `python -m map_b200.build`.
"""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libmap_b200.so")


def build_native(force=False):
    import importlib
    return importlib.import_module(__name__ + ".build").build(force=force)
