"""LDBC validation files: write a result in the format the reference's
checkers read (include/LDBC/checker.hpp), and check a result against such a
file with the same rules, so results can be compared with the published LDBC
Graphalytics outputs whenever those datasets are available.

Format: one line per vertex, "<vertex name> <value>", separated by one space.
  bfs    integer depth; unreached 9223372036854775807 (checker.hpp:52)
  sssp   distance; unreached "infinity" (checker.hpp:217); compared with a
         relative tolerance of 1e-4 (checker.hpp:226)
  pr     rank; compared with a relative tolerance of 1e-4
  wcc    the component's label (a vertex name); compared as partitions:
  cdlp   the two files must group the vertices the same way (checker.hpp:81-169)
"""
from __future__ import annotations

import math
from typing import Dict, List, Sequence, Tuple

INT32_MAX = 2**31 - 1
LLONG_MAX = 2**63 - 1
DBL_MAX = 1.7976931348623157e308


def write(path: str, kind: str, names: Sequence[str], values: Sequence) -> None:
    """values indexed by vertex id; wcc / cdlp values are vertex ids (labels)."""
    with open(path, "w") as f:
        for i, nm in enumerate(names):
            v = values[i]
            if kind == "bfs":
                s = str(LLONG_MAX) if int(v) == INT32_MAX else str(int(v))
            elif kind == "sssp":
                s = "infinity" if (not math.isfinite(float(v)) or float(v) >= DBL_MAX) else repr(float(v))
            elif kind == "pr":
                s = repr(float(v))
            elif kind in ("wcc", "cdlp"):
                s = names[int(v)]
            else:
                raise ValueError("unknown result kind %r" % kind)
            f.write("%s %s\n" % (nm, s))


def read(path: str) -> List[Tuple[str, str]]:
    out = []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            parts = line.split(" ")
            if len(parts) != 2:
                raise ValueError("validation file format error: %r" % line)
            out.append((parts[0], parts[1]))
    return out


def _partition(pairs) -> List[Tuple[str, ...]]:
    groups: Dict[str, List[str]] = {}
    for nm, lab in pairs:
        groups.setdefault(lab, []).append(nm)
    return sorted(tuple(sorted(g)) for g in groups.values())


def check(path: str, kind: str, names: Sequence[str], values: Sequence) -> Tuple[bool, str]:
    """(ok, message) of a result against a validation file, with the
    reference checkers' rules."""
    base = read(path)
    if len(base) != len(names):
        return False, "size of the validation file differs from the result"
    idx = {nm: i for i, nm in enumerate(names)}
    if kind in ("wcc", "cdlp"):
        ours = [(nm, names[int(values[i])]) for i, nm in enumerate(names)]
        if any(nm not in idx for nm, _ in base):
            return False, "validation file holds a vertex that is not in the graph"
        return (_partition(ours) == _partition(base)), "partitions compared"
    for nm, s in base:
        if nm not in idx:
            return False, "validation file holds a vertex that is not in the graph"
        v = values[idx[nm]]
        if kind == "bfs":
            b = int(s)
            if int(v) != b and not (int(v) == INT32_MAX and b == LLONG_MAX):
                return False, "%s: %s != %s" % (nm, v, s)
        elif kind == "sssp":
            if s in ("infinity", "inf"):
                if float(v) != DBL_MAX and math.isfinite(float(v)):
                    return False, "%s: %s, expected unreached" % (nm, v)
            elif abs(float(v) - float(s)) > 1e-4 * float(s):
                return False, "%s: %s != %s" % (nm, v, s)
        elif kind == "pr":
            if abs(float(v) - float(s)) > 1e-4 * abs(float(s)):
                return False, "%s: %s != %s" % (nm, v, s)
        else:
            raise ValueError("unknown result kind %r" % kind)
    return True, "values compared"
