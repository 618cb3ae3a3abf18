"""Golden text for the result-file formats (helm3d.formats), taken from the
reference's own result files under HETERO/: their names and lines, so the
tests can check file names and printf formatting byte for byte.

Run in a container that has the reference checked out:

    python tests/golden/make_formats_golden.py [reference checkout, default $HELM3D_REFERENCE or /root/reference]

writes tests/golden/formats_golden.json.
"""
import json
import os
import sys


def main(ref_root):
    hetero = None
    for dirpath, dirnames, _ in os.walk(ref_root):
        if os.path.basename(dirpath) == "HETERO":
            hetero = dirpath
            break
    if hetero is None:
        raise SystemExit("no HETERO directory under " + ref_root)
    out = {"convergence": {}, "beta": {}}
    for name in sorted(os.listdir(hetero)):
        path = os.path.join(hetero, name)
        if not os.path.isfile(path):
            continue
        with open(path) as f:
            lines = f.readlines()
        if name.startswith("convergence_"):
            out["convergence"][name] = lines
        elif name.startswith("beta_3D_norm2_") and name.endswith(".dat"):
            out["beta"][name] = lines[:12]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "formats_golden.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst, len(out["convergence"]), "logs,", len(out["beta"]), "beta files")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HELM3D_REFERENCE", "/root/reference"))
