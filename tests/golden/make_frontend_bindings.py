"""Record the ctypes signatures the reference's Python front end binds.

Usage: python tests/golden/make_frontend_bindings.py [REFERENCE_PYTHON_DIR]

Imports the unmodified reference front end (python/rakali/_core.py of the
Rakali project; the directory defaults to /root/reference/python), lets its
own loader ``_core._load_lib()`` bind this repository's librakali.so, and
writes every function it bound - symbol name, argument types and result
type as ctypes spells them - to frontend_bindings.json beside this script.
tests/test_abi_cpu.py checks the library against that record, so the check
needs no copy of the reference at test time.
"""
import ctypes
import json
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent


def type_name(t):
    if t is None:
        return "None"
    if isinstance(t, type) and issubclass(t, ctypes._Pointer):
        return f"POINTER({type_name(t._type_)})"
    return t.__name__


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/python")
    os.environ["RAKALI_LIB"] = str(ROOT / "rakali_b200" / "librakali.so")
    sys.path.insert(0, str(ref))
    from rakali import _core  # noqa: E402  (the reference's own loader)

    lib = _core._load_lib()
    out = {}
    for name, fn in sorted(vars(lib).items()):
        if isinstance(fn, ctypes._CFuncPtr):
            out[name] = {"argtypes": [type_name(t) for t in (fn.argtypes or [])],
                         "restype": type_name(fn.restype)}
    rec = {"source": "python/rakali/_core.py:88-283 (_load_lib), bound by the reference's "
                     "own loader", "working_precision_dtype": lib._rki_wp_dtype.__name__,
           "functions": out}
    (HERE / "frontend_bindings.json").write_text(json.dumps(rec, indent=1) + "\n")
    print(f"{len(out)} functions")


if __name__ == "__main__":
    main()
