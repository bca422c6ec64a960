"""sizeof / offsetof of every struct of a fp_cuda_backend.h, measured by a C
compiler: the struct blocks of this repository's include/fp_cuda_backend.h
are parsed for their field names, and a small C program that prints the
size of each struct and the offset and size of each field is compiled
against a header directory (this repository's include/, or the reference's
include/ with its fp_shared_core.h and params.h) at a bin count np = npe.

Used by tests/test_abi_layout.py and tests/golden/make_abi_layout.py."""
import os
import re
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUR_HEADER = os.path.join(ROOT, "include", "fp_cuda_backend.h")
NBS = (128, 256, 512)


def struct_fields(header=OUR_HEADER):
    """[(struct name, [field names])] of the typedef'd structs, in order."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = []
    for m in re.finditer(r"typedef\s+struct\s*\w*\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        body, name = m.group(1), m.group(2)
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            # "const double *a, *b" / "double p[np]" / "double ***logy"
            for part in decl.split(","):
                ident = re.findall(r"([A-Za-z_]\w*)\s*(?:\[[^\]]*\])?\s*$", part.strip())
                if ident:
                    fields.append(ident[0])
        out.append((name, fields))
    return out


def c_source(structs):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "fp_cuda_backend.h"', "int main(void) {"]
    for name, fields in structs:
        lines.append(f'    printf("{name} %zu\\n", sizeof({name}));')
        for f in fields:
            lines.append(f'    printf("{name}.{f} %zu %zu\\n", offsetof({name}, {f}), sizeof((({name} *)0)->{f}));')
    lines.append("    return 0;\n}")
    return "\n".join(lines) + "\n"


def measure(include_dir, nb, structs=None, cc="gcc"):
    """{key: [offset, size] or [size]} compiled against include_dir."""
    structs = structs or struct_fields()
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write(c_source(structs))
        subprocess.run([cc, "-std=gnu99", f"-Dnp={nb}", f"-Dnpe={nb}", f"-I{include_dir}", src, "-o", exe],
                       check=True, capture_output=True, text=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        key, *vals = line.split()
        res[key] = [int(v) for v in vals]
    return res


def measure_all(include_dir, structs=None):
    return {str(nb): measure(include_dir, nb, structs) for nb in NBS}
