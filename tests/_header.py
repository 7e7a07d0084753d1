"""Parsing of include/fbls_b200.h for the binding checks: the typedef'd
structs (field names and C types in order) and the function prototypes
(return and parameter types). C types are canonical strings such as
'const double *' or 'uint32_t'."""
import re
from pathlib import Path

HEADER = Path(__file__).resolve().parent.parent / "include" / "fbls_b200.h"


def c_type(text: str) -> str:
    return " ".join(text.replace("*", " * ").split())


def _text() -> str:
    return re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)


def structs() -> dict:
    out = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(fbls_\w+)\s*;", _text(), flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if decl:
                # an array field keeps its extent in the type: 'fbls_evidence_row[2]'
                m = re.fullmatch(r"(.+?)\s*\b(\w+)\s*(\[\s*\d+\s*\])?", decl, flags=re.S)
                extent = m.group(3).replace(" ", "") if m.group(3) else ""
                fields.append((m.group(2), c_type(m.group(1)) + extent))
        out[name] = fields
    return out


def prototypes() -> dict:
    out = {}
    for ret, name, params in re.findall(r"([A-Za-z_][\w\s\*]*?)\b(fbls_\w+)\s*\(([^)]*)\)\s*;", _text(), flags=re.S):
        ps = [] if params.strip() in ("", "void") else [p.strip() for p in params.split(",")]
        types = [c_type(re.fullmatch(r"(.+?)\s*\b(\w+)", p, flags=re.S).group(1)) for p in ps]
        out[name] = (c_type(ret.strip()), types)
    return out
