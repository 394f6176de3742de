"""Generate tests/golden/fft_lengths_ref.json from the reference's
util/src/FFTBestLength.cxx, read as text.

The file cannot be compiled here (it needs boost/assign); its three active
``edges += ...;`` statements are the data: the table for any parity
(``keep_odd_even`` false), then the even and the odd tables.  Commented-out
tables are skipped.

Run from the repository root:  python tests/golden/make_fft_lengths.py [reference tree]"""

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = "util/src/FFTBestLength.cxx"


def tables(text):
    code = "\n".join(line.split("//", 1)[0] for line in text.splitlines())
    found = re.findall(r"edges\s*\+=\s*([0-9,\s]+);", code)
    if len(found) != 3:
        raise SystemExit("expected three edge tables in %s, found %d" % (SRC, len(found)))
    return [[int(x) for x in f.replace("\n", " ").split(",") if x.strip()] for f in found]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WCT_REFERENCE")
    if not ref:
        raise SystemExit("usage: make_fft_lengths.py <reference tree> (or set WCT_REFERENCE)")
    with open(os.path.join(ref, SRC)) as f:
        any_, even, odd = tables(f.read())
    out = {"source": SRC, "any": any_, "even": even, "odd": odd}
    with open(os.path.join(HERE, "fft_lengths_ref.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("tables of %d, %d and %d lengths" % (len(any_), len(even), len(odd)))


if __name__ == "__main__":
    main()
