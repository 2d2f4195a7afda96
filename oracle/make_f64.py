"""Write the float64 scratch copy of the reference sources (test infrastructure).

Usage: make_f64.py <reference src dir> <output dir>

The copy is written under the oracle's git-ignored build folder only. Float
literal suffixes are stripped so constants are double, and the 4-byte phase
key of collectPhases (kernels.cpp:432-458) is widened to 8 bytes so double
offsets hash without truncation.
"""
import pathlib
import re
import sys

LITERAL = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)[fF]\b")


def main(src, dst):
    src, dst = pathlib.Path(src), pathlib.Path(dst)
    dst.mkdir(parents=True, exist_ok=True)
    for path in list(src.glob("*.cpp")) + list(src.glob("*.h")):
        text = LITERAL.sub(r"\1", path.read_text())
        if path.name == "kernels.cpp":
            text = text.replace("uint32_t offsetBits;", "uint64_t offsetBits;")
            text = text.replace("uint32_t bits;", "uint64_t bits;")
        (dst / path.name).write_text(text)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
