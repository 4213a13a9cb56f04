"""Writes the three reference headers that the SweepPatternGPU plugin (oracle/sweep_pattern_gpu.cpp) needs
changed, with the one-line additions a maintainer makes, into a scratch include folder that shadows the
reference's own (test infrastructure; the reference tree is only read).

    python oracle/plugin_headers.py <reference src folder> <output include folder>

* linear_solvers/Abstract/SweepOperator.hpp: `class SweepPatternGPU;` after the nested declaration of
  SweepPatternUniCartSequential (every sweep pattern is a nested class of SweepOperator);
* linear_solvers/Abstract/SweepCellSolve/SweepCellSolveBase.hpp: `double GetDt() const` after SetDt;
* linear_solvers/Abstract/SweepCellSolve/SweepCellSolveManager.hpp: `double GetDt() const` after SetDt.

Each insertion is anchored on a declaration that must occur exactly once; otherwise the script fails.
"""
import os
import re
import sys

EDITS = [
    ("linear_solvers/Abstract/SweepOperator.hpp",
     r"class SweepPatternUniCartSequential;",
     "    class SweepPatternGPU;   // the GPU sweep pattern (oracle/sweep_pattern_gpu.cpp)"),
    ("linear_solvers/Abstract/SweepCellSolve/SweepCellSolveBase.hpp",
     r"virtual void SetDt\( const double dt_in \);",
     "    double GetDt( void ) const {  return this->dt;  }   // read by the GPU sweep pattern"),
    ("linear_solvers/Abstract/SweepCellSolve/SweepCellSolveManager.hpp",
     r"void SetDt\( const double dt \);",
     "    double GetDt( void ) const {  return this->cell_solvers[1]->GetDt();  }   // read by the GPU sweep pattern"),
]


def main(src, out):
    for rel, anchor, line in EDITS:
        with open(os.path.join(src, rel)) as f:
            text = f.read()
        hits = [m for m in re.finditer(anchor, text)]
        if len(hits) != 1:
            raise SystemExit(f"{rel}: anchor {anchor!r} found {len(hits)} times")
        end = text.index("\n", hits[0].end()) + 1
        text = text[:end] + line + "\n" + text[end:]
        dst = os.path.join(out, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        with open(dst, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
