"""The ctypes mirrors of the C structs in include/vstark.h have the C layout
(size and field offsets as gcc lays them out)."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_header(tmp_path):
    from vortexstark_b200 import api
    mirrors = {"vs_cairo_oods_fri_io": api.CairoOodsFriIO, "vs_job": api.Job, "vs_job_result": api.JobResult}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "vstark.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        cname, field, value = line.split()
        py = mirrors[cname]
        want = C.sizeof(py) if field == "size" else getattr(py, field).offset
        assert int(value) == want, (cname, field)
