"""The Python binding's ctypes records against the C header.

Every record the C ABI takes by pointer (include/retrocam.h) has a ctypes
mirror in retrocam_b200/api.py.  A field added to one and not the other
shifts every later field: the library would read the caller's memory at
the wrong offsets.  This test compiles a small program against the header
and compares each mirrored record's size and each field's offset.
"""
import os
import subprocess
import tempfile

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RECORDS = ("rc_camera", "rc_settings", "rc_frame_desc", "rc_sppm_params", "rc_atrous_params",
           "rc_vhs_params", "rc_tuning", "rc_counters", "rc_kpcnn")


def _c_layout(records):
    """{record: (sizeof, {field: offsetof})} as the C++ compiler lays them out."""
    from retrocam_b200 import api
    lines = ["#include <cstddef>", "#include <cstdio>", '#include "retrocam.h"', "int main() {"]
    for r in records:
        lines.append(f'    std::printf("{r} . %zu\\n", sizeof({r}));')
        for f, _ in getattr(api, r)._fields_:
            lines.append(f'    std::printf("{r} {f} %zu\\n", offsetof({r}, {f}));')
    lines += ["    return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.cpp"), os.path.join(d, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "include"), src, "-o", exe], check=True,
                       capture_output=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        r, f, v = line.split()
        size, fields = layout.setdefault(r, [0, {}])
        if f == ".":
            layout[r][0] = int(v)
        else:
            fields[f] = int(v)
    return layout


@pytest.mark.parametrize("record", RECORDS)
def test_ctypes_record_matches_header(record):
    from retrocam_b200 import api
    layout = _c_layout([record])
    size, offsets = layout[record]
    cls = getattr(api, record)
    assert api.C.sizeof(cls) == size, (record, api.C.sizeof(cls), size)
    for f, _ in cls._fields_:
        assert getattr(cls, f).offset == offsets[f], (record, f, getattr(cls, f).offset, offsets[f])
