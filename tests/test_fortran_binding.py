"""The Fortran iso_c_binding module that the integration guide gives sqcalc's
maintainers (`sqc_sqnufft`), against the C ABI it binds.

No Fortran compiler exists in this image or on the GPU box, so the module is
checked by layout and by name: the fields of its `bind(c)` derived type, in
order, laid out with the companion C processor's sizes and alignments
(c_int32_t 4, c_int64_t / c_double / c_ptr 8), must sit at the offsets gcc
gives the same fields of `sqn_plan_desc` in include/sqnufft.h, with the same
total size; and every function its interface block binds by name must be
exported by libsqnufft.so.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KIND = {"integer(c_int32_t)": 4, "integer(c_int64_t)": 8, "real(c_double)": 8,
        "type(c_ptr)": 8}


def fortran_module():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```fortran\n(module sqc_sqnufft.*?end module sqc_sqnufft)\n```", text, re.S)
    assert m, "the integration guide holds the sqc_sqnufft module"
    return m.group(1)


def fortran_fields(src):
    block = re.search(r"type, bind\(c\) :: sqn_plan_desc_t\n(.*?)\n\s*end type", src, re.S)
    assert block
    fields = []
    for line in block.group(1).splitlines():
        kind, names = (s.strip() for s in line.split("::"))
        size = KIND[kind]
        for item in re.findall(r"(\w+)(?:\((\d+)\))?", names):
            name, dim = item
            fields.append((name, size, int(dim) if dim else 1))
    return fields


def c_layout(offsets_of, tmp_path):
    src = tmp_path / "layout.c"
    body = "".join('  printf("%s %%zu %%zu\\n", offsetof(sqn_plan_desc, %s), '
                   'sizeof(((sqn_plan_desc *)0)->%s));\n' % (n, n, n) for n in offsets_of)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "sqnufft.h"\n'
                   "int main(void) {\n%s"
                   '  printf("SIZE %%zu 0\\n", sizeof(sqn_plan_desc));\n  return 0;\n}\n' % body)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {name: (int(off), int(size)) for name, off, size in
            (line.split() for line in out.splitlines())}


def test_derived_type_matches_the_c_descriptor(tmp_path):
    fields = fortran_fields(fortran_module())
    got = c_layout([f[0] for f in fields], tmp_path)
    off = 0
    for name, size, dim in fields:
        off = (off + size - 1) // size * size  # natural alignment
        assert got[name] == (off, size * dim), (name, got[name], off, size * dim)
        off += size * dim
    off = (off + 7) // 8 * 8
    assert got["SIZE"][0] == off


def test_bound_functions_are_exported():
    from sqcalc_b200 import _lib
    lib = _lib.load()
    names = re.findall(r"bind\(c, name='(\w+)'\)", fortran_module())
    assert "sqn_plan_create" in names and "sqn_accumulate_frames" in names
    for n in names:
        assert hasattr(lib, n), n


@pytest.mark.parametrize("const,value", [("sqn_abi", "SQN_ABI_VERSION"),
                                         ("sqn_host", "SQN_HOST"), ("sqn_device", "SQN_DEVICE")])
def test_parameters_match_the_header(const, value):
    m = re.search(r"%s = (\d+)" % const, fortran_module())
    h = open(os.path.join(ROOT, "include", "sqnufft.h")).read()
    hv = re.search(r"#define %s (\d+)" % value, h) or re.search(r"%s = (\d+)" % value, h)
    assert m and hv and m.group(1) == hv.group(1), (const, value)
