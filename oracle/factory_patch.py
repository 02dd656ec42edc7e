"""Applies the solver-type registration of INTEGRATION.md (section 3) to copies
of the reference's src/winds/SolverFactory.h and SolverFactory.cpp, as a
maintainer would: test infrastructure for oracle/Makefile, which compiles the
result with the C++ adaptor (qes-public_b200/host/Solver_B200.*). The copies
go to the build directory given (git-ignored); the reference tree is not
touched. Each insertion checks that its anchor is present exactly once.

    python3 oracle/factory_patch.py <reference src/winds> <output dir>
"""
import os
import re
import sys


def patch(text, pattern, repl, name):
    new, n = re.subn(pattern, repl, text, count=1, flags=re.M)
    if n != 1:
        raise SystemExit(f"factory_patch: anchor for {name} not found")
    return new


def main(src, out):
    os.makedirs(out, exist_ok=True)
    h = open(os.path.join(src, "SolverFactory.h")).read()
    h = patch(h, r'^(#include "Solver\.h"\s*)$', r'\1\n#include "Solver_B200.h"', "the adaptor include")
    h = patch(h, r"(Shared_M = 4)(\s*\};)", r"\1,\n                         B200_Type = 5\2", "the B200 type")
    c = open(os.path.join(src, "SolverFactory.cpp")).read()
    c = patch(c, r'^(\s*\} else \{\s*\n\s*QESout::error\("Invalid solver type"\);)',
              "  } else if (solveType == B200_Type) {\n    solver = new Solver_B200(domain, tolerance);\n\\1",
              "the B200 branch")
    for name, text in (("SolverFactory.h", h), ("SolverFactory.cpp", c)):
        with open(os.path.join(out, name), "w") as f:
            f.write(text)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
