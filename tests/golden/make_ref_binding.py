"""Records how the reference's Python module binds libcuopus.so: for every
function it sets up, the ctypes argument and return types.  The module is
imported from the reference tree with ctypes.CDLL replaced by a recorder, so
nothing is loaded or run; the table goes to ref_binding.json and the drop-in
tests bind this repository's library (and the reference's own, built by
oracle/Makefile ref_gpu) exactly that way.

    python tests/golden/make_ref_binding.py <reference source tree>
"""
import ctypes
import importlib.util
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _name(t):
    if t is None:
        return None
    if hasattr(t, "_type_") and t.__name__.startswith("LP_"):
        return "POINTER(%s)" % _name(t._type_)
    return t.__name__


class _Fn:
    def __init__(self):
        self.argtypes = None
        self.restype = ctypes.c_int


class _Recorder:
    def __init__(self, path):
        self.fns = {}

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return self.fns.setdefault(name, _Fn())


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_ref_binding.py <reference source tree>")
    path = os.path.join(sys.argv[1], "python", "cuopus_native.py")
    spec = importlib.util.spec_from_file_location("ref_cuopus_native", path)
    mod = importlib.util.module_from_spec(spec)
    real = ctypes.CDLL
    rec = {}
    ctypes.CDLL = lambda p, *a, **k: rec.setdefault("lib", _Recorder(p))
    try:
        os.environ["CUOPUS_LIB"] = "recorder"
        spec.loader.exec_module(mod)
        mod._load()
    finally:
        ctypes.CDLL = real
    out = {n: {"argtypes": [_name(t) for t in f.argtypes], "restype": _name(f.restype)}
           for n, f in sorted(rec["lib"].fns.items())}
    with open(os.path.join(HERE, "ref_binding.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("%d functions" % len(out))


if __name__ == "__main__":
    main()
