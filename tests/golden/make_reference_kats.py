"""Extract known-answer vectors from the reference's own Catch2 unit tests.

Reads the reference test sources as text (they are never compiled or run here)
and writes ``reference_kats.json`` beside this script.  Each record keeps the
reference file and line of the REQUIRE it came from.

Covered:
  * tests/materials/mohr_coulomb_test.cc -- every ``compute_stress`` result
    (updated stress, and pdstrain where the test checks it), and every check of
    stress invariants (epsilon, rho, theta), yield functions and dF/dsigma,
    dP/dsigma made on a stress or a trial stress.
  * tests/materials/linear_elastic_test.cc -- every ``compute_stress`` result.

Catch2 runs each leaf SECTION as its own pass through the enclosing code, so
the values in force at a REQUIRE are the assignments made earlier in the
enclosing scopes; the parser keeps one scope per brace level to reproduce that.

Usage:  python tests/golden/make_reference_kats.py [reference_root]
"""
import copy
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"[-+]?(?:\d+\.?\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?)"


def strip_comments(text):
    out, i, n = [], 0, len(text)
    while i < n:
        if text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i)
            i = n if j < 0 else j + 2
        elif text[i] == '"':
            j = i + 1
            while j < n and text[j] != '"':
                j += 2 if text[j] == "\\" else 1
            out.append(text[i:j + 1])
            i = j + 1
        else:
            out.append(text[i])
            i += 1
    return "".join(out)


def statements(text):
    """Yield (kind, stmt, line) with kind in {'open','close','stmt'}."""
    buf, line, start_line, depth_paren = [], 1, 1, 0
    for ch in text:
        if ch == "\n":
            line += 1
        if ch == "(":
            depth_paren += 1
        elif ch == ")":
            depth_paren -= 1
        if depth_paren == 0 and ch in "{};":
            stmt = "".join(buf).strip()
            if ch == "{":
                yield "open", stmt, start_line
            elif ch == "}":
                if stmt:
                    yield "stmt", stmt, start_line
                yield "close", "", line
            else:
                yield "stmt", stmt, start_line
            buf = []
            start_line = line
            continue
        if not buf and ch.isspace():
            start_line = line
            continue
        buf.append(ch)


def evalnum(expr, env):
    expr = expr.strip()
    expr = re.sub(r"jmaterial\[\"(\w+)\"\]", lambda m: repr(float(env["jm"][m.group(1)])), expr)
    expr = expr.replace("std::", "")
    try:
        return float(eval(expr, {"__builtins__": {}}, {}))
    except Exception:
        return None


def parse_value(v):
    v = v.strip()
    if v == "true":
        return True
    if v == "false":
        return False
    try:
        return float(v)
    except ValueError:
        return None


def new_scope():
    return {
        "jm": {}, "dim": None, "stress": None, "dstrain": None, "state": {},
        "dvol": 0.0, "after_compute": False, "inv_arg": None, "df_arg": None,
        "tol": {},
    }


def parse_material_file(path, relpath, kind):
    text = strip_comments(open(path).read())
    stack = [new_scope()]
    stress_kats, diag_kats = [], {}
    pending = {}  # key -> record being filled (compute_stress results)
    for k, st, line in statements(text):
        cur = stack[-1]
        if k == "open":
            stack.append(copy.deepcopy(cur))
            continue
        if k == "close":
            stack.pop()
            continue
        s = " ".join(st.split())
        m = re.match(r"const unsigned Dim = (\d)", s)
        if m:
            cur["dim"] = int(m.group(1))
        m = re.match(r"const double (\w+) = (" + NUM + ")$", s)
        if m:
            cur["tol"][m.group(1)] = float(m.group(2))
        m = re.match(r'jmaterial\["(\w+)"\] = (.+)$', s)
        if m:
            val = parse_value(m.group(2))
            if val is not None:
                cur["jm"][m.group(1)] = val
            elif m.group(2).startswith('"'):
                cur["jm"][m.group(1)] = m.group(2).strip('"')
        m = re.match(r"(?:mpm::Material<Dim>::Vector6d )?(stress|dstrain|strain)\.setZero\(\)$", s)
        if m:
            cur["dstrain" if m.group(1) == "strain" else m.group(1)] = [0.0] * 6
        m = re.match(r"(stress|dstrain|strain)\((\d)\) = (" + NUM + ")$", s)
        if m:
            key = "dstrain" if m.group(1) == "strain" else m.group(1)
            if cur[key] is not None:
                cur[key][int(m.group(2))] = float(m.group(3))
        if kind == "le":
            if re.match(r"stress = material->compute_stress\(stress, strain,", s) and \
                    cur["jm"].get("stress_rate", "none") == "none":
                cur["rec_id"] = len(stress_kats)
                stress_kats.append({
                    "source": f"{relpath}:{line}", "dim": cur["dim"],
                    "material": dict(cur["jm"]), "stress": list(cur["stress"]),
                    "dstrain": list(cur["dstrain"]), "expected_stress": [None] * 6,
                    "epsilon": None,
                })
                continue
            m = re.match(r"REQUIRE\(stress\((\d)\) == Approx\((.+?)\)\.epsilon\((\w+)\)\)$", s)
            if m and "rec_id" in cur:
                rec = stress_kats[cur["rec_id"]]
                rec["expected_stress"][int(m.group(1))] = evalnum(m.group(2), cur)
                rec["epsilon"] = cur["tol"].get(m.group(3), 1e-7)
            continue
        m = re.match(r'state_variables\.at\("(\w+)"\) = (' + NUM + ")$", s)
        if m:
            cur["state"][m.group(1)] = float(m.group(2))
        m = re.search(r"assign_dvolumetric_strain\((" + NUM + r")\)", s)
        if m:
            cur["dvol"] = float(m.group(1))
        if re.search(r"initialise_state_variables\(\)", s):
            cur["state"] = {}
        m = re.search(r"compute_stress_invariants\(\s*(\w+)\s*,", s)
        if m:
            cur["inv_arg"] = m.group(1)
        m = re.search(r"compute_df_dp\(\s*\w+\s*,\s*&state_variables\s*,\s*(\w+)\s*,", s)
        if m:
            cur["df_arg"] = m.group(1)
        if re.search(r"updated_stress\s*=\s*\w+->compute_stress\(", s):
            cur["after_compute"] = True
            rec = {
                "source": f"{relpath}:{line}",
                "dim": cur["dim"],
                "material": dict(cur["jm"]),
                "stress": list(cur["stress"]),
                "dstrain": list(cur["dstrain"]),
                "dvolumetric_strain": cur["dvol"],
                "state": dict(cur["state"]),
                "expected_stress": [None] * 6,
                "expected_pdstrain": None,
                "epsilon": None,
            }
            cur["rec_id"] = len(stress_kats)
            stress_kats.append(rec)
            continue
        m = re.match(r"REQUIRE\(updated_stress\((\d)\) == Approx\((.+?)\)\.epsilon\((\w+)\)\)$", s)
        if m and "rec_id" in cur:
            rec = stress_kats[cur["rec_id"]]
            rec["expected_stress"][int(m.group(1))] = evalnum(m.group(2), cur)
            rec["epsilon"] = cur["tol"].get(m.group(3), 1e-7)
            rec.setdefault("lines", []).append(line)
            continue
        m = re.match(r'REQUIRE\(state_variables\.at\("pdstrain"\) == Approx\((.+?)\)\.epsilon\((\w+)\)\)$', s)
        if m and cur["after_compute"] and "rec_id" in cur:
            stress_kats[cur["rec_id"]]["expected_pdstrain"] = evalnum(m.group(1), cur)
            continue
        # diagnostics before compute_stress
        if cur["after_compute"]:
            continue
        m = re.match(r'REQUIRE\(state_variables\.at\("(epsilon|rho|theta)"\) == Approx\((.+?)\)\.epsilon\((\w+)\)\)$', s)
        m2 = re.match(r"REQUIRE\((yield_function(?:_trial)?)\((\d)\) == Approx\((.+?)\)\.epsilon\((\w+)\)\)$", s)
        m3 = re.match(r"REQUIRE\((df_dsigma|dp_dsigma)(?:_trial)?\((\d)\) == Approx\((.+?)\)\.epsilon\((\w+)\)\)$", s)
        if m or m2 or m3:
            arg = cur["inv_arg"] if (m or m2) else (cur["df_arg"] or cur["inv_arg"])
            if arg is None or cur["stress"] is None:
                continue
            if arg == "stress":
                sig = list(cur["stress"])
                tag = "stress"
            else:
                tag = "trial"
                sig = None
            key = (tuple(sorted(cur["jm"].items())), tuple(cur["stress"]),
                   tuple(cur["dstrain"] or []), tag,
                   tuple(sorted(cur["state"].items())), cur["dim"])
            d = diag_kats.get(key)
            if d is None:
                d = {
                    "source": f"{relpath}:{line}",
                    "dim": cur["dim"],
                    "material": dict(cur["jm"]),
                    "stress": list(cur["stress"]),
                    "dstrain": list(cur["dstrain"]) if cur["dstrain"] else None,
                    "at": tag,
                    "state": dict(cur["state"]),
                    "checks": {},
                }
                diag_kats[key] = d
            if m:
                name, val, tol = m.group(1), m.group(2), m.group(3)
            elif m2:
                name, val, tol = f"f{m2.group(2)}", m2.group(3), m2.group(4)
            else:
                name, val, tol = f"{m3.group(1)}{m3.group(2)}", m3.group(3), m3.group(4)
            d["checks"][name] = [evalnum(val, cur), cur["tol"].get(tol, 1e-7), line]
    stress_kats = [r for r in stress_kats if all(v is not None for v in r["expected_stress"])]
    return stress_kats, list(diag_kats.values())


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MPM_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_reference_kats.py <geomechanics/mpm source tree> "
                 "(or set MPM_REFERENCE_ROOT)")
    out = {"generator": "tests/golden/make_reference_kats.py"}
    mc_rel = "tests/materials/mohr_coulomb_test.cc"
    le_rel = "tests/materials/linear_elastic_test.cc"
    mc_s, mc_d = parse_material_file(os.path.join(root, mc_rel), mc_rel, "mc")
    le_s, _ = parse_material_file(os.path.join(root, le_rel), le_rel, "le")
    out["mohr_coulomb_stress"] = mc_s
    out["mohr_coulomb_diagnostics"] = mc_d
    out["linear_elastic_stress"] = le_s
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"mohr_coulomb_stress={len(mc_s)} mohr_coulomb_diagnostics={len(mc_d)} "
          f"linear_elastic_stress={len(le_s)}")


if __name__ == "__main__":
    main()
