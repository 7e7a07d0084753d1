"""The Rust binding written out in INTEGRATION.md against the C header, on
the CPU (no Rust toolchain is needed): every #[repr(C)] struct there has the
fields of the header's struct of the same name, in the same order and with
the same C types, and every extern "C" declaration has the header
prototype's parameter and return types."""
import re
from pathlib import Path

import _header as _hdr

ROOT = Path(__file__).resolve().parent.parent
DOC = ROOT / "INTEGRATION.md"

_RUST_SCALARS = {"f64": "double", "f32": "float", "u32": "uint32_t", "u64": "uint64_t", "i64": "int64_t",
                 "u8": "uint8_t", "c_int": "int", "c_char": "char", "c_void": "void"}


def _snake(name: str) -> str:
    return re.sub(r"(?<!^)([A-Z])", r"_\1", name).lower()


def _rust_type(text: str) -> str:
    """The C spelling of a Rust FFI type."""
    t = text.strip()
    a = re.fullmatch(r"\[\s*(.+?)\s*;\s*(\d+)\s*\]", t)
    if a:  # [T; N] -> T[N]
        return f"{_rust_type(a.group(1))}[{a.group(2)}]"
    m = re.fullmatch(r"\*(const|mut)\s+(.+)", t)
    if m:
        inner = _rust_type(m.group(2))
        return f"const {inner} *" if m.group(1) == "const" else f"{inner} *"
    if t in _RUST_SCALARS:
        return _RUST_SCALARS[t]
    if t.startswith("Fbls"):
        return _snake(t)
    raise AssertionError(f"unmapped Rust type {t}")


def _header():
    return _hdr.structs(), _hdr.prototypes()


def _rust_blocks():
    return re.findall(r"```rust\n(.*?)```", DOC.read_text(), flags=re.S)


def _rust():
    code = "\n".join(re.sub(r"//[^\n]*", "", b) for b in _rust_blocks())
    structs = {}
    for name, body in re.findall(r"#\[repr\(C\)\](?:\s*#\[derive\([^)]*\)\])?\s*pub struct (\w+)\s*\{(.*?)\}", code,
                                 flags=re.S):
        fields = [f.strip() for f in body.split(",") if f.strip()]
        if fields == ["_p: [u8; 0]"]:
            continue  # opaque handle
        structs[_snake(name)] = [(f.split(":", 1)[0].replace("pub", "").strip(), _rust_type(f.split(":", 1)[1]))
                                 for f in fields]
    fns = {}
    for name, params, ret in re.findall(r"pub fn (fbls_\w+)\s*\((.*?)\)\s*(?:->\s*([^;]+))?;", code, flags=re.S):
        types = [_rust_type(p.split(":", 1)[1]) for p in (x.strip() for x in params.split(",")) if p]
        fns[name] = ("void" if not ret else _rust_type(ret), types)
    return structs, fns


def test_rust_structs_match_the_header():
    cs, _ = _header()
    rs, _ = _rust()
    assert len(rs) >= 8
    for name, fields in rs.items():
        assert name in cs, name
        # the ABI is the order and the types; names may follow Rust's case (p for P)
        assert [(n.lower(), t) for n, t in fields] == [(n.lower(), t) for n, t in cs[name]], (name, fields, cs[name])


def test_rust_extern_declarations_match_the_header():
    _, cp = _header()
    _, rf = _rust()
    assert len(rf) >= 12
    for name, (ret, types) in rf.items():
        assert name in cp, name
        cret, ctypes = cp[name]
        assert ret == cret, (name, ret, cret)
        assert types == ctypes, (name, types, ctypes)
