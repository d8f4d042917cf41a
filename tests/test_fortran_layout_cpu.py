"""The Fortran interface module include/finflo_gpu.f90 against the C header.

No Fortran compiler is available, so the module is checked the way a
gfortran build would see it: its bind(C) derived types are laid out by the C
rules (which bind(C) guarantees) and compared field by field with the C
structs as gcc lays them out from include/finflo_types.h, and with the ctypes
mirrors the Python front end uses; its slot constants with enum ff_slot; and
every bind(C) name it declares must be exported by libfinflo_gpu.so.
"""
import ctypes
import os
import re
import subprocess

import pytest

from finflo_b200.case import FFParams, FFPatch, SLOT

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "finflo_gpu.f90")
SIZES = {"integer(c_int)": 4, "real(c_double)": 8}


def _f90_types():
    """{type name: [(field, kind), ...]} of the module's bind(C) types."""
    src = open(F90).read()
    out = {}
    for m in re.finditer(r"type, bind\(C\) :: (\w+)\n(.*?)end type \1", src, re.S):
        fields = []
        for line in m.group(2).splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            kind, names = line.split("::")
            kind = kind.strip()
            assert kind in SIZES, line
            fields += [(n.strip(), kind) for n in names.split(",")]
        out[m.group(1)] = fields
    return out


def _c_layout(fields):
    """Offsets and size by the C rules (natural alignment)."""
    off, offs, align = 0, {}, 1
    for name, kind in fields:
        s = SIZES[kind]
        off = (off + s - 1) // s * s
        offs[name] = off
        off += s
        align = max(align, s)
    return offs, (off + align - 1) // align * align


def _gcc_layout(tmp_path, struct, fields):
    c = tmp_path / f"layout_{struct}.c"
    body = "".join(f'  printf("%zu\\n", offsetof({struct}, {n}));\n' for n, _ in fields)
    c.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "finflo_types.h"\n'
                 f"int main(void) {{\n{body}  printf(\"%zu\\n\", sizeof({struct}));\n  return 0;\n}}\n")
    exe = tmp_path / f"layout_{struct}"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(c)])
    vals = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    return dict(zip([n for n, _ in fields], vals[:-1])), vals[-1]


@pytest.mark.parametrize("struct,mirror", [("ff_patch", FFPatch), ("ff_params", FFParams)])
def test_bind_c_types_match_the_c_structs(tmp_path, struct, mirror):
    fields = _f90_types()[struct]
    offs, size = _c_layout(fields)
    goffs, gsize = _gcc_layout(tmp_path, struct, fields)
    assert offs == goffs
    assert size == gsize == ctypes.sizeof(mirror)
    assert [n for n, _ in fields] == [n for n, _ in mirror._fields_]
    for n, _ in fields:
        assert getattr(mirror, n).offset == offs[n], n


def test_patch_carries_the_two_equation_inlet_values():
    names = [n for n, _ in _f90_types()["ff_patch"]]
    assert names[-2:] == ["bounrk", "bounep"]
    assert _c_layout(_f90_types()["ff_patch"])[1] == 120


def test_slot_constants_match_the_enum():
    src = open(F90).read()
    consts = dict((n, int(v)) for n, v in re.findall(r"\b(FF_[A-Z0-9]+) = (\d+)", src))
    slots = {k: v for k, v in consts.items() if k[3:] in SLOT or k == "FF_NSLOTS"}
    assert len(slots) >= 30
    for k, v in slots.items():
        assert v == (len(SLOT) if k == "FF_NSLOTS" else SLOT[k[3:]]), k


def test_every_bound_name_is_exported():
    from finflo_b200 import gpu
    gpu.build()
    L = ctypes.CDLL(gpu.LIB_PATH)
    names = re.findall(r'bind\(C, name="(\w+)"\)', open(F90).read())
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert L.ff_abi_version() == int(re.search(r"FF_ABI_VERSION = (\d+)", open(F90).read()).group(1))
