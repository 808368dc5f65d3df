"""The C-ABI library loads and exports every entry point include/alp_b200.h
declares (no device needed: nothing is called that touches a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        names |= set(re.findall(r"ALPB_API\s+[\w\s\*]+?\b(alpb_\w+)\s*\(", txt))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "alpb_mxv" in names and "alpb_cg_solve" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    from alp_b200 import _abi
    lib = _abi.lib()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_prototypes_cover_the_header():
    from alp_b200 import _abi
    missing = sorted(declared_symbols() - set(_abi.PROTOS))
    assert not missing, f"no ctypes prototype for: {missing}"


def test_status_strings_without_device():
    from alp_b200 import _abi
    assert _abi.lib().alpb_version() >= 1
    assert isinstance(_abi.last_error(), str)
    assert _abi.launches() >= 0


def test_only_alpb_symbols_exported():
    import subprocess
    so = ROOT / "alp_b200" / "libalp_b200.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True,
                         text=True, check=True).stdout
    syms = [l.split()[-1] for l in out.splitlines() if l.strip()]
    text_syms = [s for s in syms if not s.startswith("_") and "@" not in s]
    stray = [s for s in text_syms if not s.startswith("alpb_")]
    assert not stray, f"unexpected exports: {stray[:10]}"


def _header_declarations():
    """(name, [parameter kinds]) of every ALPB_API function in include/*.h,
    each kind "ptr" or the width and class of a scalar ("i32", "i64", ...)."""
    decls = []
    for h in sorted((ROOT / "include").glob("*.h")):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        handles = set(re.findall(r"typedef\s+struct\s+\w+\s*\*\s*(\w+)\s*;", txt))
        scalar = {"int": "i32", "int32_t": "i32", "uint32_t": "u32", "unsigned": "u32",
                  "int64_t": "i64", "uint64_t": "u64", "size_t": "u64", "double": "f64",
                  "float": "f32"}
        for name, params in re.findall(r"ALPB_API\s+[\w\s\*]+?\b(alpb_\w+)\s*\((.*?)\)\s*;", txt,
                                       flags=re.S):
            kinds = []
            params = params.strip()
            for p in ([] if params in ("", "void") else params.split(",")):
                p = " ".join(re.sub(r"\bconst\b", " ", p).split())
                if "*" in p or "[" in p:
                    kinds.append("ptr")
                    continue
                ty = " ".join(p.split()[:-1])
                kinds.append("ptr" if ty in handles else scalar.get(ty, "?" + ty))
            decls.append((name, kinds))
    return decls


def test_python_prototypes_match_header_argument_widths():
    """Every ctypes prototype passes each argument with the header's width:
    a 64-bit size sent as a 32-bit int would be read as garbage by the library."""
    import ctypes as C
    from alp_b200 import _abi
    width = {C.c_int: "i32", C.c_int32: "i32", C.c_uint32: "u32", C.c_uint: "u32",
             C.c_int64: "i64", C.c_longlong: "i64", C.c_uint64: "u64", C.c_ulonglong: "u64",
             C.c_size_t: "u64", C.c_double: "f64", C.c_float: "f32"}

    def kind(c):
        if c in (C.c_void_p, C.c_char_p) or (isinstance(c, type) and issubclass(c, C._Pointer)):
            return "ptr"
        return width.get(c, "?" + str(c))

    decls = _header_declarations()
    assert len(decls) >= 30
    bad = {}
    for name, kinds in decls:
        got = [kind(c) for c in _abi.PROTOS.get(name, [])]
        if got != kinds:
            bad[name] = (kinds, got)
    assert not bad, f"prototype and header disagree: {bad}"
