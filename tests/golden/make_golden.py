"""Extract the reference's own known-answer values for this path into reference_goldens.json.

Reads the kete sources (read-only) as text and pulls the literal expected values out of
their unit tests, so the committed fixture can be traced line by line:

* kete_core/src/propagation/radau.rs:356-374      basic_two_body (Radau + central_accel)
* kete_core/src/propagation/kepler.rs:444-476     parabolic / hyperbolic universal Kepler
* src/tests/flux/test_model.py:37-51              WISE NEATM fluxes
* kete_core/src/fitting/newton.rs:72-78           Newton-Raphson root

Usage: python tests/golden/make_golden.py [path/to/kete]
"""
import json
import os
import re
import sys

NUM = r"-?\d+(?:\.\d+)?(?:e-?\d+)?"


def grab(text, pattern, n=None):
    vals = [float(v) for v in re.findall(pattern, text)]
    if n is not None and len(vals) < n:
        raise SystemExit(f"pattern {pattern!r} matched {len(vals)} values, expected {n}")
    return vals


def main(root):
    core = os.path.join(root, "src", "kete_core", "src")
    radau = open(os.path.join(core, "propagation", "radau.rs")).read()
    kepler = open(os.path.join(core, "propagation", "kepler.rs")).read()
    model = open(os.path.join(root, "src", "tests", "flux", "test_model.py")).read()

    t = radau[radau.index("fn basic_two_body"):]
    # explicit extraction keeps the sign convention of each assert
    asserts = re.findall(r"\((pos|vel)\[(\d)\] ([+-]) (" + NUM + r")\)\.abs\(\) < (" + NUM + r")", t)
    radau_golden = {"asserts": []}
    for which, idx, sign, val, tol in asserts:
        expected = -float(val) if sign == "+" else float(val)
        radau_golden["asserts"].append([which, int(idx), expected, float(tol)])
    vec = re.search(r"Vector3::new\((" + NUM + r"), (" + NUM + r"), 0\.\)\s*,\s*Vector3::new\((" +
                    NUM + r"), (" + NUM + r"), 0\.\)", t)
    radau_golden["pos0"] = [float(vec.group(1)), float(vec.group(2)), 0.0]
    radau_golden["vel0"] = [float(vec.group(3)), float(vec.group(4)), 0.0]
    radau_golden["t1"] = 1000.0

    def kep(name):
        s = kepler[kepler.index(f"fn {name}"):]
        s = s[: s.index("#[test]") if "#[test]" in s else len(s)]
        pos = re.search(r"let pos_exp = Vector3::new\((" + NUM + "), (" + NUM + ")", s)
        vel = re.search(r"let vel_exp = (-?)Vector3::new\((" + NUM + "), (" + NUM + ")", s)
        sgn = -1.0 if vel.group(1) == "-" else 1.0
        return {"pos_exp": [float(pos.group(1)), float(pos.group(2)), 0.0],
                "vel_exp": [sgn * float(vel.group(2)), sgn * float(vel.group(3)), 0.0]}

    m = model[model.index("def test_wise_neatm_model"):]
    fluxes = [float(v) for v in re.findall(r"np\.isclose\(output\.fluxes\[\d\], (" + NUM + r")\)", m)]
    out = {
        "source": "values copied from the kete test suite; see make_golden.py for file:line",
        "radau_basic_two_body": radau_golden,
        "kepler_parabolic": kep("test_kepler_parabolic"),
        "kepler_hyperbolic": kep("test_kepler_hyperbolic"),
        "wise_neatm": {"sun2obj": [1, 1, 0], "sun2obs": [0, 1, 0], "vis_albedo": 0.3,
                       "band_albedos": [0.3, 0.3, 0.3, 0.3], "g_param": 0.15, "beaming": 1.4,
                       "diam": 1.0, "fluxes": fluxes},
        "newton": {"root": 1.0, "tol": 1e-12},
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KETE_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <path to the kete reference checkout> "
                 "(or set KETE_REFERENCE_ROOT)")
    main(root)
