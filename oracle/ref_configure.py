"""Write the configuration headers SymPhas's sources include, from SymPhas's
own templates, for the oracle's pin (oracle/ref.mk).  TEST INFRASTRUCTURE ONLY.

SymPhas's CMake fills `@VAR@` and `#cmakedefine NAME` in seven `*.in`
templates (configured-defs.h.in, lib/lib-defs.h.in, io/io-defs.h.in,
sol/inc/stencildefs.h.in, io/inc/plottername.h.in, io/inc/readincludes.h.in,
io/inc/writeincludes.h.in).  This script does the same substitutions for one
fixed configuration, so no CMake runs:

- modules lib, datatypes, sym, sol, io (USE_IO=ON; no conf, no proc);
- THREAD_COUNT 2, VECTOR_TYPE_NAME VectorValue (lib/CMakeLists.txt:41-42);
- every optional feature off: FFTW, MPI, CUDA, timing printouts, LaTeX,
  xdrfile, VTK, stencil overrides, all-stencils and stencil generation (the
  basic-stencils default, sol/CMakeLists.txt AVAILABLE_STENCILS_BASIC_ONLY);
- AVAILABLE_DIMENSIONS 2,3; accuracy 2 (2D and 3D) and 4 (2D); the stencil
  point lists of sol/CMakeLists.txt.

Usage: python ref_configure.py <symphas source dir> <output dir>
"""
import os
import re
import sys

ON = {"USING_IO"}  # every other #cmakedefine is left undefined

VALUES = {
    "THREAD_COUNT": "2",
    "VECTOR_TYPE_NAME": "VectorValue",
    "GNU_PLOTTER": "qt",
    "AVAILABLE_DIMENSIONS": "2,3",
    "CONFIGURED_DEF_FILES": '#include "lib-defs.h"\n#include "io-defs.h"',
    "WRITE_STENCIL_OVERRIDE_DEFINITIONS": "",
}

POINTS = {  # sol/CMakeLists.txt AVAILABLE_STENCIL_POINTS_*
    ("LAPLACIAN", 2): "5,9", ("GRADLAPLACIAN", 2): "6,8,12,16", ("BILAPLACIAN", 2): "13,17,21",
    ("LAPLACIAN", 3): "7,15,19,21,27", ("GRADLAPLACIAN", 3): "10,12,28,36,40",
    ("BILAPLACIAN", 3): "21,25,41,52,57",
}
ACCURACY = {2: "2,4", 3: "2"}


def _guarded(name, value=""):
    return "\n#ifndef %s\n#define %s%s\n#endif\n" % (name, name, (" " + value) if value else "")


def stencil_values():
    pts, order, acc = "", "", ""
    for dim in (2, 3):
        for op in ("LAPLACIAN", "GRADLAPLACIAN", "BILAPLACIAN"):
            pts += _guarded("AVAILABLE_%s_POINTS_%dD" % (op, dim), POINTS[(op, dim)])
        order += _guarded("ORDER_LIST_%dD" % dim, ACCURACY[dim])
        for a in ACCURACY[dim].split(","):
            acc += _guarded("ORDER_LIST_%dD_HAS_%sH" % (dim, a))
    return {"WRITE_STENCIL_POINT_DEFINITIONS": pts, "WRITE_ORDER_DEFINITIONS": order,
            "WRITE_ORDER_ACCURACY_DEFINITIONS": acc}


TEMPLATES = [
    ("configured-defs.h.in", "configured-defs.h"),
    ("lib/lib-defs.h.in", "lib-defs.h"),
    ("io/io-defs.h.in", "io-defs.h"),
    ("sol/inc/stencildefs.h.in", "stencildefs.h"),
    ("io/inc/plottername.h.in", "plottername.h"),
    ("io/inc/readincludes.h.in", "readincludes.h"),
    ("io/inc/writeincludes.h.in", "writeincludes.h"),
]


def configure(text, values):
    def cmakedefine(m):
        return "#define %s" % m.group(1) if m.group(1) in ON else "/* #undef %s */" % m.group(1)

    text = re.sub(r"#cmakedefine\s+(\w+)[^\n]*", cmakedefine, text)

    def at(m):
        if m.group(1) not in values:
            raise KeyError("no value for @%s@" % m.group(1))
        return values[m.group(1)]

    return re.sub(r"@(\w+)@", at, text)


def main(src, out):
    os.makedirs(out, exist_ok=True)
    values = dict(VALUES)
    values.update(stencil_values())
    for tin, tout in TEMPLATES:
        with open(os.path.join(src, tin)) as f:
            text = configure(f.read(), values)
        path = os.path.join(out, tout)
        if not text.endswith("\n"):
            text += "\n"
        old = open(path).read() if os.path.exists(path) else None
        if old != text:  # keep the time stamp when nothing changed
            with open(path, "w") as f:
                f.write(text)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
