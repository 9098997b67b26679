"""Regenerate the golden fixtures in tests/golden/ from the reference checkout.

Run where the reference is present (the GPU test machine does not have it;
the generated JSON files are committed and travel with the repository):

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Outputs
* isaac_golden.json     -- verbatim copy of tests/fixtures/isaac/golden.json
  (ISAAC states after irandinit and after one round; flam3 isaac.c).
* variations_flam3.json -- the 99 flam3-instrumented f64 (tx, ty) -> (x, y)
  fixture files of tests/fixtures/variations/, with each row's parameters
  resolved to the packed param0..param9 slots (src/serialize.ts
  VARIATION_PARAMS order) and the affine coefficients / injected parameters
  that src/variations.test.ts feeds each runner.  `runner` records how the
  reference test checks the file: "det" (deterministic), "affine",
  "branch" (RNG branch unknown: any of `branches` outcomes may match),
  "julia" (two branches), "smoke" (RNG placeholder values, shape only).
"""
from __future__ import annotations

import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _call_text(src: str, start: int) -> str:
    i = src.index("(", start)
    depth = 0
    for j in range(i, len(src)):
        depth += {"(": 1, ")": -1}.get(src[j], 0)
        if depth == 0:
            return src[i + 1:j]
    raise ValueError("unbalanced call")


def _dict_literal(text: str) -> dict:
    m = re.search(r"\{([^{}]*)\}", text)
    if not m:
        return {}
    out = {}
    for k, v in re.findall(r"(\w+)\s*:\s*([-+0-9.eE]+)", m.group(1)):
        out[k] = float(v)
    return out


def main(ref: str) -> None:
    shutil.copyfile(os.path.join(ref, "tests/fixtures/isaac/golden.json"),
                    os.path.join(HERE, "isaac_golden.json"))

    catalog = json.load(open(os.path.join(REPO, "pyr3_b200", "catalog.json")))
    by_name = {v["name"]: v for v in catalog["variations"]}
    test_src = open(os.path.join(ref, "src/variations.test.ts")).read()

    runners = {}
    for m in re.finditer(r"describe\('variation: (\w+)", test_src):
        name = m.group(1)
        body_end = test_src.find("describe(", m.end())
        body = test_src[m.end(): body_end if body_end > 0 else len(test_src)]
        rm = re.search(r"(runDeterministic|runWithAffine|runMultiBranchRng|runJulia|runSmoke)\s*\(", body)
        if not rm:
            continue
        kind = rm.group(1)
        args = _call_text(body, rm.start())
        injected = _dict_literal(args)
        branches = None
        if kind == "runMultiBranchRng":
            nums = re.findall(r"fix,\s*(\d+)", args)
            branches = int(nums[0]) if nums else None
        runners[name] = (kind, injected, branches)

    kinds = {"runDeterministic": "det", "runWithAffine": "affine",
             "runMultiBranchRng": "branch", "runJulia": "julia", "runSmoke": "smoke"}
    out = []
    fixdir = os.path.join(ref, "tests/fixtures/variations")
    for fn in sorted(os.listdir(fixdir)):
        fx = json.load(open(os.path.join(fixdir, fn)))
        vname = fx["variation"]
        cat = by_name.get(vname) or by_name.get({"oscilloscope": "oscilloscope"}.get(vname, vname))
        if cat is None:
            raise KeyError(f"fixture {fn}: variation {vname} not in catalog")
        kind, injected, branches = runners.get(vname, ("runDeterministic", {}, None))
        affine = {k: v for k, v in injected.items() if k in "abcdef" and len(k) == 1}
        params = list(cat["defaults"]) + [0.0] * (10 - len(cat["defaults"]))
        for slot, pname in enumerate(cat["params"]):
            for key, val in injected.items():
                if key.endswith("_" + pname):
                    params[slot] = val
        rows = []
        for r in fx["fixtures"]:
            if r.get("params"):
                for slot, pname in enumerate(cat["params"]):
                    for key, val in r["params"].items():
                        if key == pname or key.endswith("_" + pname):
                            params[slot] = float(val)
            rows.append([r["tx"], r["ty"], r["weight"], r["expected_x"], r["expected_y"]])
        out.append({
            "name": vname, "idx": cat["idx"], "runner": kinds[kind],
            "branches": branches, "affine": affine, "params": params, "rows": rows,
        })
    with open(os.path.join(HERE, "variations_flam3.json"), "w") as f:
        json.dump(out, f, indent=0, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {len(out)} variation fixture sets")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYR3_REFERENCE")
    if not root:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT (or set PYR3_REFERENCE)")
    main(root)
