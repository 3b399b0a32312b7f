"""The C-ABI library loads and exports every function include/*.h declares
(no device calls)."""
import re
import subprocess
from pathlib import Path

import zigtrace_b200._native as N

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(zt_[a-z_0-9]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_binding_list():
    assert declared_functions() == set(N.SIGNATURES)


def test_library_exports_every_declared_symbol(native_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared_functions() - exported
    assert not missing, missing
    for name in declared_functions():
        assert getattr(native_lib, name) is not None


def test_version_and_error_string(native_lib):
    assert native_lib.zt_version().startswith(b"zigtrace-b200")
    assert native_lib.zt_scene_build(None) == -5
    assert b"NULL" in native_lib.zt_last_error()


def _header_arity():
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "zigtrace_b200.h").read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"(zt_[a-z_0-9]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_zig_binding_declarations_match_the_header():
    """INTEGRATION.md's Zig binding cannot be compiled here (no Zig
    toolchain): its extern declarations are held to the header instead --
    every function it declares exists with the same number of parameters."""
    doc = (ROOT / "INTEGRATION.md").read_text()
    decls = re.findall(r"extern fn (zt_[a-z_0-9]+)\((.*?)\)\s*[^;]*;", doc, flags=re.S)
    assert len(decls) >= 10
    header = _header_arity()
    for name, args in decls:
        assert name in header, name
        n = 0 if not args.strip() else len([a for a in args.split(",") if a.strip()])
        assert n == header[name], (name, n, header[name])
