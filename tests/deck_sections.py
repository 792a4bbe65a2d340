"""Result sections of a nec2++-style text output, read the way the
reference's regression comparison (nec2diff, src/necDiff.cpp with
AntennaInput.h, PowerBudget.h, RadiationInput.h) reads them, plus the
near-field tables: lists of numeric rows per section instance."""
import re

_NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[Ee][-+]?\d+)?")


def _numbers(line):
    return [float(x) for x in _NUM.findall(line)]


def sections(text):
    lines = text.splitlines()
    out = {"inputs": [], "budgets": [], "patterns": [], "near": []}
    k = 0
    while k < len(lines):
        line = lines[k]
        if "ANTENNA INPUT PARAMETERS" in line:
            while "(WATTS)" not in lines[k]:
                k += 1
            k += 1
            rows = []
            while k < len(lines) and lines[k].strip():
                rows.append(_numbers(lines[k].replace("*", " ")))
                k += 1
            out["inputs"].append(rows)
            continue
        if "POWER BUDGET" in line:
            vals = []
            k += 1
            while len(vals) < 5 and k < len(lines):
                if "=" in lines[k]:
                    vals.append(_numbers(lines[k].split("=", 1)[1])[0])
                k += 1
            out["budgets"].append(vals)
            continue
        if "RADIATION PATTERNS" in line:
            while "VOLTS/M" not in lines[k]:
                k += 1
            k += 1
            rows = []
            while k < len(lines) and lines[k].strip():
                rows.append(_numbers(lines[k]))
                k += 1
            out["patterns"].append(rows)
            continue
        if "NEAR ELECTRIC FIELDS" in line or "NEAR MAGNETIC FIELDS" in line:
            kind = 0 if "ELECTRIC" in line else 1
            while "METERS    METERS" not in lines[k]:
                k += 1
            k += 1
            rows = []
            while k < len(lines) and lines[k].strip():
                rows.append(_numbers(lines[k]))
                k += 1
            out["near"].append((kind, rows))
            continue
        k += 1
    return out


def rel_diff(a, b):
    """nec2diff's relative difference (BaseInput.h diff): |a-b| / |a+b|,
    values below 1e-8 in magnitude equal."""
    if a == b or (abs(a) < 1e-8 and abs(b) < 1e-8):
        return 0.0
    s = abs(a + b)
    return abs(a - b) / s if s else abs(a - b)
