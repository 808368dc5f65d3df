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
