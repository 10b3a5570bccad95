"""Extract the reference's golden R-matrix outputs into a committed JSON fixture.

Run in a container that has the HPRMAT sources mounted (read-only) at
``/root/reference``:

    python tests/golden/make_golden.py [/root/reference]

It reads Descouvemont's example inputs and printed outputs,
``rmat_pierre/Ex{1,2,3,4,5}/data*`` and ``rmat_pierre/Ex{1,2,3,4,5}/output*.txt`` (the files the
HPRMAT README compares its solvers against, README.md:113-121), the wave functions the drivers
write for their rmax < 0 card (``rmat_pierre/Ex{1,2,3,4,5}/wf*.txt``) and Ex3's wf_print output,
and writes ``tests/golden/reference_examples.json``.  Nothing else is transformed: the numbers are
the printed 5-significant-digit values.  The physics inputs of each example (potential
forms, masses, charges) are restated by the tests from the example drivers
(``examples/Ex{1,2,4}/example*_hp.f90``, ``rmat_pierre/Ex3/example3.f``); only the mesh/energy cards and printed results
come from here.
"""
from __future__ import annotations

import json
import os
import re
import sys

NUM = r"[-+]?\d+\.\d+E[-+]\d+"


def parse_data(path, with_print_mesh=False):
    """Input cards: (j, nr, ns, rmax), for Ex3 then (npoin, h), followed by (ne, e0, estep)
    lines."""
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
        extra = {}
        if with_print_mesh:
            extra = {"npoin": int(lines[i][0]), "h": float(lines[i][1])}
            i += 1
        energies = []
        while i < len(lines):
            ne, e0, es = int(lines[i][0]), float(lines[i][1]), float(lines[i][2])
            i += 1
            if ne == 0:
                break
            energies.append((ne, e0, es))
        cards.append({"j": j, "nr": nr, "ns": ns, "rmax": rmax, "energies": energies, **extra})
    return cards


def parse_data_ex5(path):
    """Ex5 cards: (nr, rmax) then (ne, e0, estep) lines; l = 0, ns = 1 in the driver."""
    cards = []
    with open(path) as f:
        lines = [ln.split("!")[0].split() for ln in f if ln.strip()]
    i = 0
    while i < len(lines):
        nr, rmax = int(lines[i][0]), float(lines[i][1])
        if nr == 0:
            break
        i += 1
        energies = []
        while i < len(lines):
            ne, e0, es = int(lines[i][0]), float(lines[i][1]), float(lines[i][2])
            i += 1
            if ne == 0:
                break
            energies.append((ne, e0, es))
        cards.append({"j": 0, "nr": nr, "ns": 1, "rmax": rmax, "energies": energies})
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


def parse_wavefunctions(path):
    """Blocks of the drivers' wave_functions.txt (rmat_pierre/Ex*/wf*.txt): per energy the
    internal wave functions at the mesh points (r, then Re/Im per channel) and the external
    ones at r = zrma(nr ns) + 0.2 i, i = 0..11."""
    blocks = []
    part = None
    with open(path) as f:
        for ln in f:
            m = re.match(r"\s*Wave function, E=\s*([-\d.]+)\s+entrance channel=\s*(\d+)", ln)
            if m:
                blocks.append({"E": float(m.group(1)), "entrance": int(m.group(2)), "internal": [], "external": []})
                continue
            if "Internal wave functions" in ln:
                part = "internal"
                continue
            if "External wave functions" in ln:
                part = "external"
                continue
            vals = re.findall(NUM, ln)
            if vals and blocks:
                r = float(ln.split()[0])
                blocks[-1][part].append([r] + [float(v) for v in vals])
    return blocks


def parse_fixed_step(path):
    """wf_print output of Ex3 (rmat_pierre/Ex3/output3.txt): after each energy of the card that
    asks for it, per channel the rows (r, Re, Im) on the uniform mesh."""
    out = []
    energy = None
    cur = None
    with open(path) as f:
        for ln in f:
            m = re.match(r"E \(MeV\)=\s*([-\d.]+)", ln)
            if m:
                energy = float(m.group(1))
            if "Wave function at a fixed step size" in ln:
                cur = {"E": energy, "channels": []}
                out.append(cur)
                continue
            if re.match(r"\s*Channel\s+\d+", ln) and cur is not None:
                cur["channels"].append([])
                continue
            vals = re.findall(NUM, ln)
            if cur is not None and cur["channels"] and len(vals) == 2 and "E (MeV)" not in ln:
                cur["channels"][-1].append([float(ln.split()[0])] + [float(v) for v in vals])
    return out


def main(ref):
    out = {"source": "rmat_pierre/Ex{1,2,3,4,5}/output*.txt, wf*.txt and data* of HPRMAT", "examples": {}}
    spec = {
        "ex1": ("Ex1", "data1", "output1.txt", ["Collision matrix="]),
        "ex2": ("Ex2", "data2", "output2.txt", ["phase shift (rad.)="]),
        "ex3": ("Ex3", "data3", "output3.txt", ["Amplitude=", "phase shift (rad.)="]),
        "ex4": ("Ex4", "data4", "output4.txt", ["Amplitude=", "phase shift (rad.)="]),
        "ex5": ("Ex5", "data5", "output5.txt", ["phase shift (deg.)="]),
    }
    out["wavefunctions"] = {}
    for name, (d, data, outp, keys) in spec.items():
        if name == "ex5":
            cards = parse_data_ex5(os.path.join(ref, "rmat_pierre", d, data))
        else:
            cards = parse_data(os.path.join(ref, "rmat_pierre", d, data), with_print_mesh=(name == "ex3"))
        wf = os.path.join(ref, "rmat_pierre", d, "wf" + name[-1] + ".txt")
        if os.path.exists(wf):
            # written by the card with rmax < 0 (twf = .true. in the drivers)
            out["wavefunctions"][name] = {"card": [i for i, c in enumerate(cards) if c["rmax"] < 0][0],
                                          "blocks": parse_wavefunctions(wf)}
        res = {}
        for key in keys:
            res[key] = parse_output(os.path.join(ref, "rmat_pierre", d, outp), key)
        for ic, card in enumerate(cards):
            for key in keys:
                card.setdefault("printed", {})[key] = res[key][ic]["rows"]
        out["examples"][name] = cards
    out["fixed_step"] = {"ex3": parse_fixed_step(os.path.join(ref, "rmat_pierre", "Ex3", "output3.txt"))}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_examples.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
