"""The Python binding (fbls_b200/_native.py) against the C ABI, on the CPU:
every ctypes signature has the header prototype's parameter and return
types, and every ctypes Structure has the size and field offsets that gcc
gives the header's struct of the same name (a small C program prints
sizeof and offsetof for every field)."""
import ctypes as C
import json
import shutil
import subprocess

import pytest

import _header
from fbls_b200 import _native as N

# ctypes class -> the C spellings it passes (c_int64 and c_longlong are one class where long is 64-bit)
_SCALARS = {}
for _ct, _names in ((C.c_double, {"double"}), (C.c_float, {"float"}), (C.c_int, {"int"}),
                    (C.c_uint32, {"uint32_t"}), (C.c_int64, {"int64_t"}), (C.c_longlong, {"long long"}),
                    (C.c_uint64, {"uint64_t"}), (C.c_uint8, {"uint8_t"})):
    _SCALARS.setdefault(_ct, set()).update(_names)
_STRUCTS = {N.Bank: "fbls_bank", N.Row: "fbls_row", N.ScanStats: "fbls_scan_stats", N.Config: "fbls_config",
            N.EvidenceRow: "fbls_evidence_row", N.Counters: "fbls_counters", N.Star: "fbls_star",
            N.MapJob: "fbls_map_job", N.PrepConfig: "fbls_prep_config", N.FamilyOut: "fbls_family_out",
            N.EventStats: "fbls_event_stats", N.EvidenceJob: "fbls_evidence_job", N.Tuning: "fbls_tuning"}


def _base(c_type: str) -> str:
    return c_type.replace("const ", "").replace(" *", "").strip()


def _matches(ct, c_type: str) -> bool:
    """Does ctypes type `ct` pass the C type `c_type` (constness aside)?"""
    pointer = c_type.endswith("*")
    if ct is C.c_void_p:
        return pointer  # an opaque handle, device pointer or stream
    if ct is C.c_char_p:
        return _base(c_type) == "char" and pointer
    if isinstance(ct, type) and issubclass(ct, C._Pointer):
        target = ct._type_
        if target is C.c_void_p:  # pointer to a handle: fbls_ready** and the like
            return c_type.count("*") == 2
        names = {_STRUCTS[target]} if target in _STRUCTS else _SCALARS.get(target, set())
        return pointer and c_type.count("*") == 1 and _base(c_type) in names
    return not pointer and c_type in _SCALARS.get(ct, set())


def test_signatures_match_the_prototypes():
    protos = _header.prototypes()
    assert set(N.SIGNATURES) == set(protos)
    for name, (res, args) in N.SIGNATURES.items():
        cret, cparams = protos[name]
        assert len(args) == len(cparams), name
        for i, (ct, c) in enumerate(zip(args, cparams)):
            assert _matches(ct, c), (name, i, ct, c)
        if res is None:
            assert cret == "void", name
        else:
            assert _matches(res, cret), (name, res, cret)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_structure_layouts_match_gcc(tmp_path):
    structs = _header.structs()
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "fbls_b200.h"', "int main(void) {",
             '    printf("{");']
    first = True
    for name, fields in structs.items():
        parts = [f'\\"{name}\\": [%zu'] + [", %zu"] * len(fields) + ["]"]
        args = [f"sizeof({name})"] + [f"offsetof({name}, {f})" for f, _ in fields]
        lines.append(f'    printf("{"" if first else ", "}{"".join(parts)}", {", ".join(args)});')
        first = False
    lines += ['    printf("}\\n");', "    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    include = _header.HEADER.parent
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", f"-I{include}", str(src), "-o", str(exe)], check=True)
    layout = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    assert set(_STRUCTS.values()) <= set(layout)
    for cls, name in _STRUCTS.items():
        size, offsets = layout[name][0], layout[name][1:]
        assert C.sizeof(cls) == size, name
        assert [f for f, _ in cls._fields_] == [f for f, _ in structs[name]], name
        assert [getattr(cls, f).offset for f, _ in cls._fields_] == offsets, name
