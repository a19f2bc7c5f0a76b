"""Build the golden fixtures of the test suite from the reference project (run once, here).

Inputs (read-only, reference project):
  data/{cellcycle,sizek,metastasis,Montagud2022_Prostate_Cancer}.{bnd,cfg}  example models
  test/*.res   stdout dumps (UTF-16) of the reference's `visualize` output for those models

Outputs (committed):
  tests/golden/models/<name>.bnd, .cfg   the example models, unchanged
  tests/golden/<name>.res.json           the .res dumps parsed into
      {"final": {state: prob}, "fixed": {state: prob},
       "windows": [{"begin": a, "end": b, "entropy": H, "transition_entropy": TH,
                    "probs": {state: prob}}]}
    State names use the older "-" separator of the dumps; tests compare them as sets of nodes.

usage: python tests/golden/make_fixtures.py /path/to/reference
"""
import json
import os
import shutil
import sys

MODELS = ["cellcycle", "sizek", "metastasis", "Montagud2022_Prostate_Cancer"]


def parse_res(text: str) -> dict:
    out = {"final": {}, "fixed": {}, "windows": []}
    section = None
    cur = None
    for line in text.splitlines():
        line = line.strip()
        if not line:
            continue
        if line == "final points:":
            section = "final"
            continue
        if line == "fixed points:":
            section = "fixed"
            continue
        if line.startswith("window ("):
            a, b = line[len("window ("):-1].split(",")
            cur = {"begin": float(a), "end": float(b), "probs": {}}
            out["windows"].append(cur)
            section = "window"
            continue
        if line.startswith("entropy:"):
            cur["entropy"] = float(line.split(":")[1])
            continue
        if line.startswith("transition entropy:"):
            cur["transition_entropy"] = float(line.split(":")[1])
            continue
        prob, name = line.split(" ", 1)
        target = out[section] if section in ("final", "fixed") else cur["probs"]
        target[name] = float(prob)
    return out


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <reference checkout> (the directory holding data/ and test/)")
    ref = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "models"), exist_ok=True)
    for name in MODELS:
        for ext in ("bnd", "cfg"):
            shutil.copyfile(os.path.join(ref, "data", f"{name}.{ext}"), os.path.join(here, "models", f"{name}.{ext}"))
        raw = open(os.path.join(ref, "test", f"{name}.res"), "rb").read()
        parsed = parse_res(raw.decode("utf-16"))
        with open(os.path.join(here, f"{name}.res.json"), "w") as f:
            json.dump(parsed, f, indent=0, sort_keys=True)
        print(name, len(parsed["windows"]), "windows,", len(parsed["final"]), "final,", len(parsed["fixed"]), "fixed")


if __name__ == "__main__":
    main()
