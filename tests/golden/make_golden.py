"""Regenerates the golden fixtures in this folder from the reference checkout.

Run where a reference checkout is available, naming its root either as the
argument or in the REFERENCE_ROOT environment variable:
    python tests/golden/make_golden.py /path/to/reference

It copies
  * js_fdtd/results/out.json -- the only reference-produced Float64 output: the
    200-step ``ifa-fr4-substrate`` run (V trace, S11 at 500 frequencies and the
    xy/xz directivity cuts at 2.0/5.0 GHz) -- into ``ref_out_ifa_fr4_200.json``,
    keeping only the numeric payload (the timestamp is dropped);
  * the four scenario files js_fdtd/scenarios/*.json into ``scenarios/`` (the
    inputs that produced and that go with that output).
Nothing at test time reads the reference checkout; the tests read these files.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "js_fdtd", "results", "out.json")
    with open(src) as f:
        d = json.load(f)
    meta = dict(d["meta"])
    meta.pop("generated", None)
    out = {
        "source": "js_fdtd/results/out.json",
        "meta": meta,
        "sparams": d["sparams"],
        "farfield": [{k: v for k, v in ff.items() if k != "angles_deg"} for ff in d["farfield"]],
        "voltages": [{"label": v["label"], "values": v["values"]} for v in d["timeDomain"]["voltages"]],
    }
    with open(os.path.join(HERE, "ref_out_ifa_fr4_200.json"), "w") as f:
        json.dump(out, f)
    sdir = os.path.join(ref_root, "js_fdtd", "scenarios")
    os.makedirs(os.path.join(HERE, "scenarios"), exist_ok=True)
    for name in sorted(os.listdir(sdir)):
        if name.endswith(".json"):
            with open(os.path.join(sdir, name)) as f:
                scn = json.load(f)
            with open(os.path.join(HERE, "scenarios", name), "w") as f:
                json.dump(scn, f, indent=1)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set REFERENCE_ROOT)")
    main(root)
