"""ctypes binding of ``liblmm_b200.so`` (the C ABI declared in include/*.h).

The argument and return types of every entry point are read from the
declarations in ``include/lmm_c.h`` (and the other headers there), so the
binding cannot drift from the header and pointers are never truncated.
``call(name, *args)`` raises ``LmmError`` carrying ``lmm_last_error_string()``
on a non-zero status.  There is no fallback: importing this module fails if
the CUDA library has not been built.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

_PKG = Path(__file__).resolve().parent
ROOT = _PKG.parent
LIB_PATH = _PKG / "liblmm_b200.so"
HEADERS = sorted((ROOT / "include").glob("*.h"))

_SCALARS = {
    "int": ctypes.c_int,
    "uint32_t": ctypes.c_uint32,
    "unsigned": ctypes.c_uint,
    "float": ctypes.c_float,
    "double": ctypes.c_double,
    "size_t": ctypes.c_size_t,
    "long": ctypes.c_long,
    "lmm_stream_t": ctypes.c_void_p,
}

_DECL = re.compile(
    r"^\s*(?P<ret>(?:const\s+)?[A-Za-z_][\w]*\s*\**)\s*(?P<name>lmm_\w+)\s*\((?P<args>[^;{]*?)\)\s*;",
    re.M | re.S,
)


def _ctype(decl: str):
    decl = re.sub(r"/\*.*?\*/", " ", decl).strip()
    if "*" in decl:
        if re.match(r"^\s*const\s+char\s*\*", decl) and "(" not in decl:
            return ctypes.c_char_p
        return ctypes.c_void_p
    words = [w for w in re.split(r"\s+", decl) if w and w != "const"]
    if not words:
        raise ValueError(f"cannot parse parameter {decl!r}")
    if words[:3] == ["unsigned", "long", "long"]:
        return ctypes.c_ulonglong
    if words[:2] == ["long", "long"]:
        return ctypes.c_longlong
    if words[:2] == ["unsigned", "long"]:
        return ctypes.c_ulong
    base = words[0]
    if base not in _SCALARS:
        raise ValueError(f"unsupported C type {base!r} in {decl!r}")
    return _SCALARS[base]


def parse_headers(paths=None) -> dict[str, tuple[object, list]]:
    """name -> (restype, [argtypes]) for every ``lmm_*`` declaration."""
    sigs: dict[str, tuple[object, list]] = {}
    for path in paths or HEADERS:
        text = re.sub(r"/\*.*?\*/", " ", Path(path).read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        for m in _DECL.finditer(text):
            ret = m.group("ret").strip()
            restype = ctypes.c_char_p if ("char" in ret and "*" in ret) else _ctype(ret)
            args = m.group("args").strip()
            argtypes = [] if args in ("", "void") else [_ctype(a) for a in args.split(",")]
            sigs[m.group("name")] = (restype, argtypes)
    return sigs


SIGNATURES = parse_headers()


class LmmError(RuntimeError):
    """A C-ABI entry point returned a non-zero status."""

    def __init__(self, name: str, status: int, message: str):
        super().__init__(f"{name} failed with status {status}: {message}")
        self.status = status


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m useful_code_b200.build_ext` "
            "(the CUDA library is required; there is no CPU fallback)"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()


def call(name: str, *args) -> int:
    """Call ``name`` and raise ``LmmError`` on a non-zero status."""
    st = getattr(LIB, name)(*args)
    if st != 0:
        msg = LIB.lmm_last_error_string().decode(errors="replace")
        raise LmmError(name, st, msg)
    return st
