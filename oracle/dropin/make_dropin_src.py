"""TEST INFRASTRUCTURE ONLY: the reference sources with the drop-in hooks.

    python oracle/dropin/make_dropin_src.py <reference dir> <output dir>

Copies the reference engine's top-level sources (*.hh, *.cc) into the output
folder (a build folder under oracle/_ref/, never committed) and makes the
reference's two DP entry points begin with a call into dmst_dropin.hh, which
answers them through libdummest_b200.so and returns:

  findSimilaritiesBackwardOnly  dummest-dp-backward.hh (the filter wave)
  findSimilarities              dummest-search.hh (survivor wave, calibration)

Nothing else of the reference changes.  The script finds each function
definition by its name and checks its parameter names, and fails if either
is not found as expected.
"""
from __future__ import annotations

import glob
import os
import re
import shutil
import sys

HOOKS = {
    "dummest-dp-backward.hh": (
        "findSimilaritiesBackwardOnly",
        ["bestScores", "profile", "decoded", "scratch", "activeCount"],
        "dmst_dropin::backwardOnly(bestScores, profile, decoded, activeCount);",
    ),
    "dummest-search.hh": (
        "findSimilarities",
        ["similarities", "profile", "decoded", "minProbRatio", "scratch", "activeCount", "filterBestOut",
         "needAlign"],
        "dmst_dropin::similarities(similarities, profile, decoded, minProbRatio, activeCount, filterBestOut);",
    ),
}


def _param_names(params: str) -> list[str]:
    names, depth, cur = [], 0, ""
    for ch in params + ",":
        if ch in "<([":
            depth += 1
        elif ch in ">)]":
            depth -= 1
        if ch == "," and depth == 0:
            decl = cur.split("=")[0].strip()
            names.append(re.findall(r"[A-Za-z_]\w*", decl)[-1])
            cur = ""
        else:
            cur += ch
    return names


def hook(text: str, func: str, params: list[str], call: str, path: str) -> str:
    # the definition: "void func(" at the start of a line, its parameter list, then "{"
    m = None
    for cand in re.finditer(r"^void\s+" + re.escape(func) + r"\s*\(", text, flags=re.M):
        depth, i = 1, cand.end()
        while depth:
            depth += {"(": 1, ")": -1}.get(text[i], 0)
            i += 1
        rest = text[i:].lstrip()
        if rest.startswith("{"):
            m = (cand.start(), cand.end(), i, i + (len(text[i:]) - len(rest)))
            break
    if m is None:
        raise SystemExit(f"{path}: no definition of {func}")
    start, popen, pclose, brace = m
    got = _param_names(text[popen:pclose - 1])
    if got != params:
        raise SystemExit(f"{path}: {func} takes ({', '.join(got)}), expected ({', '.join(params)})")
    body = brace + 1
    return (text[:start] + '#include "dmst_dropin.hh"\n' + text[start:body] + "\n    " + call + "\n    return;\n"
            + text[body:])


def main(reference: str, out: str) -> None:
    os.makedirs(out, exist_ok=True)
    for f in glob.glob(os.path.join(reference, "*.hh")) + glob.glob(os.path.join(reference, "*.cc")):
        shutil.copyfile(f, os.path.join(out, os.path.basename(f)))
    for name, (func, params, call) in HOOKS.items():
        path = os.path.join(out, name)
        text = open(path).read()
        open(path, "w").write(hook(text, func, params, call, path))


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    main(sys.argv[1], sys.argv[2])
