"""Regenerate the golden fixtures in this directory from the reference's own
unit-test vectors (test/unit/*.json of Julienbxl/Zyklop).

The reference tests load these JSON files at run time
(test/unit/test_fp_bn254.cu, test_fr_bn254.cu, test_ntt.cu, test_msm.cu,
test_msm_g2.cu).  This script re-encodes them compactly (every 4 x u64
little-endian element becomes one hex integer) and keeps a bounded subset of
the 10 004 Fp inverse cases so the fixtures stay small.  Nothing is computed
here: every expected value is copied from the reference's vectors.

    python tests/golden/make_fixtures.py [REFERENCE_ROOT]
"""
import json
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ZK_REFERENCE_DIR", "/root/reference")
UNIT = os.path.join(REF, "test", "unit")
OUT = os.path.dirname(os.path.abspath(__file__))


def h(limbs):
    """4 little-endian u64 limbs (ints or decimal strings) -> hex integer."""
    v = 0
    for i, x in enumerate(limbs):
        v |= int(x) << (64 * i)
    return hex(v)


def fp_vectors():
    d = json.load(open(os.path.join(UNIT, "test_vectors.json")))
    out = {"meta": d["meta"], "by_mm64_check": d["by_mm64_check"]}
    for op in ("fp_add", "fp_sub", "fp_mul"):
        out[op] = [[h(v["a"]), h(v["b"]), h(v["r"])] for v in d[op]]
    for op in ("fp_neg", "fp_sqr"):
        out[op] = [[h(v["a"]), h(v["r"])] for v in d[op]]
    # fp_inv works on canonical values (test_fp_bn254.cu:255-280); keep the
    # first 600 (they include the edge cases listed first) and every 50th.
    inv = d["fp_inv"]
    keep = inv[:600] + inv[600::50]
    out["fp_inv"] = [[h(v["a"]), h(v["r"])] for v in keep]
    out["curve_g1"] = [
        {"note": v.get("note", ""),
         "p1": [h(v["p1"][0]), h(v["p1"][1])],
         "p2": [h(v["p2"][0]), h(v["p2"][1])],
         "r": [h(v["r"][0]), h(v["r"][1])]}
        for v in d["curve_g1"] if "p1" in v and "p2" in v
    ]
    # k * G cases: canonical affine result of scalar * generator
    out["curve_g1_mul"] = [
        {"note": v.get("note", ""), "scalar": hex(int(v["scalar"])) if not isinstance(v["scalar"], list) else h(v["scalar"]),
         "r": [h(v["r"][0]), h(v["r"][1])]}
        for v in d["curve_g1"] if "scalar" in v
    ]
    return out


def fr_vectors():
    d = json.load(open(os.path.join(UNIT, "test_vectors_fr.json")))
    out = {"r": d["r"], "R_Fr": h(d["R_Fr"]), "R2_Fr": h(d["R2_Fr"]), "ops": {}}
    for v in d["vectors"]:
        op = v["op"]
        rec = {}
        for k, x in v.items():
            if k == "op":
                continue
            if isinstance(x, list) and len(x) == 4:
                rec[k] = h(x)
            else:
                rec[k] = x
        out["ops"].setdefault(op, []).append(rec)
    return out


def ntt_vectors():
    d = json.load(open(os.path.join(UNIT, "test_vectors_ntt.json")))
    return [{"log_n": v["log_n"], "desc": v["desc"],
             "input": [h(x) for x in v["input"]],
             "expected": [h(x) for x in v["expected"]]} for v in d]


def msm_g1_vectors():
    d = json.load(open(os.path.join(UNIT, "test_vectors_msm.json")))
    return [{"label": v["label"], "N": v["N"],
             "px": [h(x) for x in v["Px"]], "py": [h(x) for x in v["Py"]],
             "scalars": [h(x) for x in v["scalars"]],
             "out": [h(v["out_x"]), h(v["out_y"])]} for v in d]


def msm_g2_vectors():
    d = json.load(open(os.path.join(UNIT, "test_vectors_msm_g2.json")))
    res = []
    for v in d:
        o = v["out"]
        res.append({
            "label": v["label"], "N": v["N"],
            "px": [[h(x["a0"]), h(x["a1"])] for x in v["Px"]],
            "py": [[h(x["a0"]), h(x["a1"])] for x in v["Py"]],
            "scalars": [h(x) for x in v["scalars"]],
            "infinity": bool(o.get("infinity", False)),
            "out": [h(o["x"]["a0"]), h(o["x"]["a1"]), h(o["y"]["a0"]), h(o["y"]["a1"])],
        })
    return res


def main():
    files = {
        "fp_vectors.json": fp_vectors(),
        "fr_vectors.json": fr_vectors(),
        "ntt_vectors.json": ntt_vectors(),
        "msm_g1_vectors.json": msm_g1_vectors(),
        "msm_g2_vectors.json": msm_g2_vectors(),
    }
    for name, obj in files.items():
        with open(os.path.join(OUT, name), "w") as f:
            json.dump(obj, f, separators=(",", ":"))
        print(name, os.path.getsize(os.path.join(OUT, name)))


if __name__ == "__main__":
    main()
