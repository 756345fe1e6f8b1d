"""The C-ABI's three descriptions agree: include/ntcfd.h (compiled with gcc
to print every struct's size and field offsets), the ctypes structures of
ntustcfdlab_b200/abi.py, and the bind(C) derived types and interfaces of
fortran/ntcfd_iface.f90 (parsed; no Fortran compiler is installed)."""
import ctypes
import os
import re
import subprocess

import pytest

from ntustcfdlab_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "fortran", "ntcfd_iface.f90")

STRUCTS = {
    "ntcfd_params": abi.NtcfdParams,
    "ntcfd_step_info": abi.NtcfdStepInfo,
    "ntcfd_kernel_times": abi.NtcfdKernelTimes,
    "ntcfd_adj_spec": abi.NtcfdAdjSpec,
    "ntcfd_adj_result": abi.NtcfdAdjResult,
}

F_KIND = {"c_int": 4, "c_double": 8, "c_float": 4, "c_long_long": 8}


def _ctypes_fields(cls):
    out = []
    for name, typ in cls._fields_:
        n, t = 1, typ
        while hasattr(t, "_length_"):
            n *= t._length_
            t = t._type_
        out.append((name.lower(), ctypes.sizeof(t), n, getattr(cls, name).offset))
    return out


def _fortran_types():
    src = open(F90).read()
    types = {}
    for m in re.finditer(r"type, bind\(C\) :: (\w+)\n(.*?)end type", src, re.S):
        fields = []
        for line in m.group(2).splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            d = re.match(r"(integer|real)\((\w+)\) :: (.*)", line)
            assert d, line
            size = F_KIND[d.group(2)]
            for item in re.findall(r"(\w+)(\([\d, ]+\))?", d.group(3)):
                name, dims = item
                n = 1
                if dims:
                    for x in dims.strip("()").split(","):
                        n *= int(x)
                fields.append((name.lower(), size, n))
        types[m.group(1)] = fields
    return types


def _c_layout(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ntcfd.h"', "int main(void) {"]
    for s, cls in STRUCTS.items():
        lines.append(f'printf("{s} size %zu\\n", sizeof({s}));')
        for name, *_ in cls._fields_:
            lines.append(f'printf("{s} {name} %zu\\n", offsetof({s}, {name}));')
    lines.append("return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        s, f, v = line.split()
        res[(s, f)] = int(v)
    return res


def test_ctypes_structs_match_the_compiled_header(tmp_path):
    lay = _c_layout(tmp_path)
    for s, cls in STRUCTS.items():
        assert lay[(s, "size")] == ctypes.sizeof(cls), s
        for name, *_ in cls._fields_:
            assert lay[(s, name)] == getattr(cls, name).offset, (s, name)


def test_fortran_types_match_ctypes():
    ftypes = _fortran_types()
    assert set(ftypes) == set(STRUCTS)
    for s, cls in STRUCTS.items():
        cf = [(n, sz, cnt) for n, sz, cnt, _ in _ctypes_fields(cls)]
        assert ftypes[s] == cf, s
        # bind(C) layout: natural alignment of each field, size rounded to the largest
        off = al = 0
        for _, sz, cnt in ftypes[s]:
            off = (off + sz - 1) // sz * sz + sz * cnt
            al = max(al, sz)
        assert (off + al - 1) // al * al == ctypes.sizeof(cls), s


def test_fortran_interfaces_cover_every_entry_point(ntcfd_lib):
    names = set(re.findall(r'bind\(C, name="(\w+)"\)', open(F90).read()))
    assert names == set(abi.SIGNATURES)
    for n in names:
        assert hasattr(ntcfd_lib, n)
