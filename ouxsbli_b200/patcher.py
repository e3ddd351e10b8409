"""Text patcher for fypp macro lines and Fortran parameter declarations.

Same behaviour as the reference's ``ouxsbli.patch`` (ouxsbli/patcher.py:7-151):
``#:set NAME = value`` lines and ``..., parameter :: name = expr`` lines are
rewritten in place; names not found are appended as ``#:set`` lines only when
the text is a fypp file.  Kept for users that maintain reference case
directories; the B200 Case API itself needs no source patching.
"""
from __future__ import annotations

import re

__all__ = ["patch"]


def _to_fortran_double(v: float) -> str:
    """1600.0 -> '1600.0d0', 1e-5 -> '1d-05' (10 significant digits)."""
    s = f"{v:.10g}"
    if "e" in s or "E" in s:
        return s.replace("e", "d").replace("E", "d")
    if "." not in s:
        s += ".0"
    return s + "d0"


def _split_comment(line: str) -> tuple[str, str]:
    if "!" in line:
        at = line.index("!")
        return line[:at], line[at:]
    return line, ""


def _is_macro_line(line: str, name: str) -> bool:
    return re.search(r"^\s*#:\s*set\s+" + re.escape(name) + r"\b", line, re.IGNORECASE) is not None


def _is_param_line(line: str, name: str) -> bool:
    code = line.split("!")[0]
    return re.search(r"parameter\s*::\s*" + re.escape(name) + r"\b", code, re.IGNORECASE) is not None


def _macro_value(value) -> str:
    if isinstance(value, bool):
        return "True" if value else "False"
    if isinstance(value, int):
        return str(value)
    if isinstance(value, float):
        return _to_fortran_double(value)
    if isinstance(value, str):
        v = value.strip()
        quoted = len(v) >= 2 and v[0] == v[-1] and v[0] in "'\""
        return v if quoted else f"'{v}'"
    return str(value)


def _param_value(value) -> str:
    if isinstance(value, bool):
        return ".true." if value else ".false."
    if isinstance(value, int):
        return str(value)
    if isinstance(value, float):
        return _to_fortran_double(value)
    return str(value)


def _rewrite_macro(line: str, name: str, value) -> str:
    code, comment = _split_comment(line)
    new = re.sub(r"(#:\s*set\s+" + re.escape(name) + r"\s*=\s*)(.+?)\s*$",
                 lambda m: m.group(1) + _macro_value(value), code, flags=re.IGNORECASE)
    if new == code and "=" in code:
        new = code.split("=")[0] + "= " + _macro_value(value)
    return new + comment


def _rewrite_param(line: str, name: str, value) -> str:
    code, comment = _split_comment(line)
    new = re.sub(r"(parameter\s*::\s*" + re.escape(name) + r"\s*=\s*).*$",
                 lambda m: m.group(1) + _param_value(value), code, flags=re.IGNORECASE)
    return new + comment


def patch(src_text: str, changes: dict) -> str:
    """Return src_text with each `changes` entry applied (see module docstring)."""
    lines = src_text.splitlines()
    for i, line in enumerate(lines):
        for name, value in changes.items():
            if _is_macro_line(line, name):
                lines[i] = _rewrite_macro(line, name, value)
                break
            if _is_param_line(line, name):
                lines[i] = _rewrite_param(line, name, value)
                break
    if any("#:set" in ln for ln in lines):
        for name, value in changes.items():
            if not any(_is_macro_line(ln, name) or _is_param_line(ln, name) for ln in lines):
                lines.append(_rewrite_macro(f"#:set {name} = ", name, value))
    return "\n".join(lines) + "\n"
