"""Helpers for the tests of the drop-in C++ interface (focalors_poisson_b200/cpp/): writes golden composite
cases in the text format of tests/cases/composite_case.cpp, builds and runs that driver, parses its output."""
import os
import subprocess

import numpy as np

from golden_io import composite_case
from focalors_poisson_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER_SRC = os.path.join(HERE, "cases", "composite_case.cpp")


def driver(tmpdir) -> str:
    return build.compile_driver(DRIVER_SRC, os.path.join(str(tmpdir), "composite_case"))


def write_case(path, name, tol=None):
    geo, rhs, ghosts, _, (m, case_tol, it), _ = composite_case(name)
    nd = len(geo["nx"])
    lines = [str(nd)]
    for d in range(nd):
        lines.append(" ".join([str(geo["nx"][d]), str(geo["ny"][d]), repr(geo["hx"][d]), repr(geo["hy"][d])]
                              + [str(b) for b in geo["bc"][d]]))
    lines.append(str(len(geo["connections"])))
    lines += [" ".join(str(v) for v in c) for c in geo["connections"]]
    lines.append(f"{m} {repr(case_tol if tol is None else tol)} {it}")
    blocks = []
    if ghosts is not None:
        for d in range(nd):
            for f in range(4):
                if ghosts[d][f] is not None:
                    blocks.append(f"{d} {f}\n" + "\n".join(repr(float(v)) for v in np.ravel(ghosts[d][f])))
    lines.append(str(len(blocks)))
    lines += blocks
    for r in rhs:
        lines.append("\n".join(repr(float(v)) for v in np.ravel(r)))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return geo


def run(exe, case_path, tree_only=False, timeout=300):
    cmd = [exe, case_path] + (["--tree-only"] if tree_only else [])
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)


def parse(stdout, geo):
    """(root, levels per domain, fields or None) from the driver's output."""
    root, levels, fields, cur, vals = None, {}, {}, None, []
    for line in stdout.splitlines():
        if line.startswith("root "):
            root = int(line.split()[1])
        elif line.startswith("level "):
            k = int(line.split()[1].rstrip(":"))
            for d in line.split(":")[1].split():
                levels[int(d)] = k
        elif line.startswith("field "):
            if cur is not None:
                fields[cur] = vals
            cur, vals = int(line.split()[1]), []
        elif cur is not None and line.strip():
            vals.append(float(line))
    if cur is not None:
        fields[cur] = vals
    nd = len(geo["nx"])
    out = None
    if fields:
        out = [np.asarray(fields[d]).reshape(geo["nx"][d], geo["ny"][d]) for d in range(nd)]
    return root, [levels.get(d, -1) for d in range(nd)], out


def parse_printed_blocks(stdout):
    """Fields printed by field2::print (rows of comma-separated values), split at the reference drivers'
    separator lines ('----...' and 'Testing ...')."""
    blocks, cur = [], []
    for line in stdout.splitlines():
        if (line.strip() and set(line.strip()) == {"-"}) or line.startswith("Testing"):
            if cur:
                blocks.append(np.asarray(cur))
            cur = []
            continue
        if line.strip():
            cur.append([float(v) for v in line.split(",")])
    if cur:
        blocks.append(np.asarray(cur))
    return blocks
