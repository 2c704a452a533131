"""The Fortran side of the boundary against the C header: the bind(C) derived
types of mrm_b200/shim/mrm_gpu_m.f90 (mrm_geom_t, mrm_stats_t) must lay out
exactly as mrm_geom and mrm_gpu_stats of include/mrm_gpu.h, field by field.

No Fortran compiler exists here, so the Fortran layout is computed from the
declarations by the interoperability rules of ISO_C_BINDING (each component
at the next offset aligned to its C type, arrays in column-major order with
the same element count as the C array) and compared with offsetof / sizeof
from a C program compiled against the header.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "mrm_b200", "shim", "mrm_gpu_m.f90")
HEADER_DIR = os.path.join(ROOT, "include")
KIND_BYTES = {"C_INT32_T": 4, "C_INT": 4, "C_DOUBLE": 8, "C_INT64_T": 8}
TYPES = {"mrm_geom_t": "mrm_geom", "mrm_stats_t": "mrm_gpu_stats"}


def _fortran_types():
    src = open(SHIM).read()
    params = {m.group(1): int(m.group(2)) for m in re.finditer(r"integer,\s*parameter\s*::\s*(\w+)\s*=\s*(\d+)", src)}
    types = {}
    for m in re.finditer(r"type,\s*bind\(C\)\s*::\s*(\w+)\s*\n(.*?)\n\s*end type", src, re.S):
        fields = []
        for line in m.group(2).splitlines():
            d = re.match(r"\s*(?:integer|real)\((\w+)\)\s*::\s*(.*)", line)
            if not d:
                continue
            kind = d.group(1)
            for name, dims in re.findall(r"(\w+)(?:\(([^)]*)\))?", d.group(2)):
                count = 1
                for dim in (dims.split(",") if dims else []):
                    dim = dim.strip()
                    count *= params[dim] if dim in params else int(dim)
                fields.append((name, KIND_BYTES[kind], count))
        types[m.group(1)] = fields
    return types, params


def _layout(fields):
    out, off, align = {}, 0, 1
    for name, size, count in fields:
        off = (off + size - 1) // size * size
        out[name] = (off, size * count)
        off += size * count
        align = max(align, size)
    return out, (off + align - 1) // align * align


def test_bind_c_types_match_header(tmp_path):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    types, params = _fortran_types()
    assert set(types) == set(TYPES), types.keys()
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "mrm_gpu.h"', "int main(void) {",
             '  printf("MAXL %d\\n", MRM_MAX_LAYERS);']
    for ft, ct in TYPES.items():
        lines.append(f'  printf("{ct} sizeof %zu\\n", sizeof({ct}));')
        for name, _, _ in types[ft]:
            lines.append(f'  printf("{ct} {name} %zu %zu\\n", offsetof({ct}, {name}), sizeof((({ct}*)0)->{name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "layout")
    subprocess.run([gcc, "-I", HEADER_DIR, str(src), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines()
    c = {}
    for line in out:
        parts = line.split()
        if parts[0] == "MAXL":
            assert int(parts[1]) == params["MAXL"], "MAXL of the shim differs from MRM_MAX_LAYERS"
        elif parts[1] == "sizeof":
            c[(parts[0], "sizeof")] = int(parts[2])
        else:
            c[(parts[0], parts[1])] = (int(parts[2]), int(parts[3]))
    for ft, ct in TYPES.items():
        lay, size = _layout(types[ft])
        # every C field appears in the Fortran type, in the same order and place
        for name, (off, nbytes) in lay.items():
            assert c[(ct, name)] == (off, nbytes), (ct, name, c[(ct, name)], (off, nbytes))
        assert c[(ct, "sizeof")] == size, (ct, c[(ct, "sizeof")], size)
        assert len(lay) == sum(1 for k in c if k[0] == ct and k[1] != "sizeof")


def test_shim_source_form_and_bound_names():
    """Free-form Fortran lines are at most 132 characters, and every bind(C)
    name of the shim is a function the C header declares."""
    import re
    src = open(SHIM).read()
    for k, line in enumerate(src.splitlines(), 1):
        assert len(line) <= 132, f"line {k} has {len(line)} characters"
    header = open(os.path.join(ROOT, "include", "mrm_gpu.h")).read()
    bound = re.findall(r'bind\(C,\s*name="(\w+)"\)', src)
    assert bound
    for name in bound:
        assert re.search(r"\b" + name + r"\s*\(", header), name
