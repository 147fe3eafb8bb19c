"""Generates the golden fixtures in this folder from the reference's own test inputs.

Usage: python make_golden.py <path of a Forte checkout>.  Reads the
FCIDUMP integral files of tests/methods/integrals-fcidump-{1..6} and stores them as compact
npz fixtures, together with the reference energies those tests assert
(tests/methods/integrals-fcidump-N/input.dat: ``reffci``) and the active-space settings of
their input decks.  The fixtures are what tests/ reads; nothing at test time touches the
reference checkout.
"""
import os
import re
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python make_golden.py <path of a Forte checkout>")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))


def parse_dump(path):
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    hdr = []
    while True:
        i += 1
        if "END" in lines[i]:
            break
        hdr.append(lines[i])
    data = np.array([list(map(float, ln.split())) for ln in lines[i + 1:] if ln.strip()])
    return "\n".join(hdr), data


def main():
    for k in range(1, 7):
        d = os.path.join(REF, "tests", "methods", f"integrals-fcidump-{k}")
        inp = open(os.path.join(d, "input.dat")).read()
        ref = float(re.search(r"reffci\s*=\s*([-0-9.eE+]+)", inp).group(1))

        def lst(key):
            m = re.search(key + r"\s*\[([^\]]*)\]", inp)
            return np.array([int(x) for x in m.group(1).split(",")]) if m else np.zeros(0, int)

        def num(key):
            m = re.search(r"\n\s*" + key + r"\s+([0-9]+)", inp)
            return int(m.group(1)) if m else -1

        hdr, data = parse_dump(os.path.join(d, "INTDUMP"))
        idx = data[:, 1:].astype(np.int8)
        vals = data[:, 0]
        same = 0
        for j in range(1, k):  # tests that share an INTDUMP store it once
            prev = np.load(os.path.join(HERE, f"fcidump{j}.npz"))
            if "values" in prev and str(prev["header"]) == hdr and np.array_equal(prev["values"], vals) \
                    and np.array_equal(prev["index"], idx):
                same = j
                break
        extra = dict(integrals_from=same) if same else dict(values=vals, index=idx)
        np.savez_compressed(
            os.path.join(HERE, f"fcidump{k}.npz"),
            header=np.array(hdr), reffci=ref, **extra,
            frozen_docc=lst("frozen_docc"), restricted_docc=lst("restricted_docc"),
            active=lst("active"), nel=num("nel"), multiplicity=num("multiplicity"))
        print(k, ref, data.shape)


if __name__ == "__main__":
    main()
