"""Extract the reference's golden R-matrix outputs into a committed JSON fixture.

Run in a container that has the HPRMAT sources mounted (read-only) at
``/root/reference``:

    python tests/golden/make_golden.py [/root/reference]

It reads Descouvemont's example inputs and printed outputs,
``rmat_pierre/Ex{1,2,4}/data*`` and ``rmat_pierre/Ex{1,2,4}/output*.txt`` (the files the
HPRMAT README compares its solvers against, README.md:113-121), and writes
``tests/golden/reference_examples.json``.  Nothing else is transformed: the numbers are
the printed 5-significant-digit values.  The physics inputs of each example (potential
forms, masses, charges) are restated by the tests from the example drivers
(``examples/Ex{1,2,4}/example*_hp.f90``); only the mesh/energy cards and printed results
come from here.
"""
from __future__ import annotations

import json
import os
import re
import sys

NUM = r"[-+]?\d+\.\d+E[-+]\d+"


def parse_data(path):
    """Input cards: (j, nr, ns, rmax) followed by (ne, e0, estep) lines, Ex1/2/4 layout."""
    cards = []
    with open(path) as f:
        lines = [ln.split("!")[0].split() for ln in f if ln.strip()]
    i = 0
    while i < len(lines):
        head = lines[i]
        if int(head[0]) < 0:
            break
        j, nr, ns, rmax = int(head[0]), int(head[1]), int(head[2]), float(head[3])
        i += 1
        energies = []
        while i < len(lines):
            ne, e0, es = int(lines[i][0]), float(lines[i][1]), float(lines[i][2])
            i += 1
            if ne == 0:
                break
            energies.append((ne, e0, es))
        cards.append({"j": j, "nr": nr, "ns": ns, "rmax": rmax, "energies": energies})
    return cards


def parse_output(path, key):
    """Printed result lines after ``key`` (e.g. 'Collision matrix='), continuation lines included."""
    blocks = []
    cur = None
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        ln = lines[i]
        m = re.match(r"\s*total angular momentum=\s*(\d+)", ln)
        if m:
            cur = {"j": int(m.group(1)), "rows": []}
            blocks.append(cur)
        m = re.match(r"E \(MeV\)=\s*([-\d.]+)\s*" + re.escape(key) + r"(.*)$", ln)
        if m and cur is not None:
            vals = [float(v) for v in re.findall(NUM, m.group(2))]
            k = i + 1
            while k < len(lines) and re.match(r"^\s+" + NUM, lines[k]) and "E (MeV)" not in lines[k]:
                vals += [float(v) for v in re.findall(NUM, lines[k])]
                k += 1
            cur["rows"].append({"E": float(m.group(1)), "values": vals})
        i += 1
    return blocks


def main(ref):
    out = {"source": "rmat_pierre/Ex{1,2,4}/output*.txt and data* of HPRMAT", "examples": {}}
    spec = {
        "ex1": ("Ex1", "data1", "output1.txt", ["Collision matrix="]),
        "ex2": ("Ex2", "data2", "output2.txt", ["phase shift (rad.)="]),
        "ex4": ("Ex4", "data4", "output4.txt", ["Amplitude=", "phase shift (rad.)="]),
    }
    for name, (d, data, outp, keys) in spec.items():
        cards = parse_data(os.path.join(ref, "rmat_pierre", d, data))
        res = {}
        for key in keys:
            res[key] = parse_output(os.path.join(ref, "rmat_pierre", d, outp), key)
        for ic, card in enumerate(cards):
            for key in keys:
                card.setdefault("printed", {})[key] = res[key][ic]["rows"]
        out["examples"][name] = cards
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_examples.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
