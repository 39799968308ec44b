"""Regenerate tests/golden/mg25.json from the reference's own example files.

Reads (from the reference checkout given as argv[1], a required argument):
  examples/sd/sd.sps            orbits (isospin format)
  examples/sd/usdb.int          USDB interaction (63 TBMEs + 3 SPEs)
  examples/sd/input.mg25ref     4 protons, 5 neutrons, 2Jz = 1, scaling 1 18 25 0.3
  examples/sd/input.mg25altwfn  same nucleus, scaling 0 1 1 1 (xspe = 0)
  examples/sd/output/mg25ref.res, mg25alt.res   10 lowest energies, J, T (5 decimals) and
                                                every one-body density block (5 decimals)
  examples/sd/output/mg25dx_dres.m              the same density blocks to 8 decimals
  examples/sd/output/mg25expectH.res, overlap.dat
                                                <H> of the mg25ref states (6 decimals) and the
                                                overlaps of mg25ref state 1 with mg25alt's states
  examples/sd/sdspin.opme, output/mg25spinstrength1.res
                                                the spin operator and the strength function
                                                of the mg25ref ground state (input.mg25strength)
and writes the numbers as JSON.  Run once in a checkout that has the reference;
the JSON is what the tests read (the reference is not needed at test time).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from bigstickpublick_b200 import model  # noqa: E402


def read_res(path):
    states = []
    lines = open(path).read().splitlines()
    for i, ln in enumerate(lines):
        if "State" in ln and "E" in ln and "Ex" in ln:
            for row in lines[i + 1:]:
                f = row.split()
                if len(f) != 5 or not f[0].isdigit():
                    break
                states.append({"n": int(f[0]), "E": float(f[1]), "Ex": float(f[2]), "J": float(f[3]),
                               "T": float(f[4])})
            break
    m = re.search(r"(\d+)\s+iterations", open(path).read())
    return states, int(m.group(1)) if m else None


def read_diag_density(path):
    """Jt=0, Tt=0 one-body densities rho(a,b) of the blocks whose initial and
    final state coincide: {state: [[a, b, rho_T0, rho_T1], ...], 'J2': 2J}"""
    lines = open(path).read().splitlines()
    out = {}
    i = 0
    while i < len(lines):
        m = re.match(r"\s*Initial state #\s+(\d+).*2xJ, 2xT =\s+(\d+)\s+(\d+)", lines[i])
        if m and i + 1 < len(lines):
            f = re.match(r"\s*Final state\s+#\s+(\d+)", lines[i + 1])
            if f and f.group(1) == m.group(1) and "Jt =   0, Tt = 0" in lines[i + 2]:
                rows = []
                for row in lines[i + 3:]:
                    t = row.split()
                    if len(t) != 4 or not t[0].isdigit():
                        break
                    rows.append([int(t[0]), int(t[1]), float(t[2]), float(t[3])])
                out[m.group(1)] = {"J2": int(m.group(2)), "T2": int(m.group(3)), "rho": rows}
        i += 1
    return out


def read_all_densities(path):
    """Every one-body density block the reference prints: initial and final
    state (number, 2J, 2T), Jt, and the rows [a, b, rho_Tt=0, rho_Tt=1]."""
    lines = open(path).read().splitlines()
    blocks = []
    i = 0
    while i < len(lines):
        m = re.match(r"\s*Initial state #\s+(\d+).*2xJ, 2xT =\s+(\d+)\s+(\d+)", lines[i])
        f = re.match(r"\s*Final state\s+#\s+(\d+).*2xJ, 2xT =\s+(\d+)\s+(\d+)", lines[i + 1]) \
            if m and i + 1 < len(lines) else None
        if not f:
            i += 1
            continue
        i += 2
        while i < len(lines):
            jt = re.match(r"\s*Jt =\s+(\d+), Tt = 0\s+1", lines[i])
            if not jt:
                break
            rows = []
            i += 1
            while i < len(lines):
                t = lines[i].split()
                if len(t) != 4 or not t[0].isdigit():
                    break
                rows.append([int(t[0]), int(t[1]), float(t[2]), float(t[3])])
                i += 1
            blocks.append({"i": int(m.group(1)), "J2i": int(m.group(2)), "T2i": int(m.group(3)),
                           "f": int(f.group(1)), "J2f": int(f.group(2)), "T2f": int(f.group(3)),
                           "Jt": int(jt.group(1)), "rho": rows})
    return blocks


def read_strength(path):
    """Total strength, iteration count and the (energy, strength) table of a
    strength-function .res file."""
    lines = open(path).read().splitlines()
    out = {"total": None, "iterations": None, "table": []}
    for i, ln in enumerate(lines):
        m = re.match(r"\s*([0-9.Ee+-]+)\s+= total strength", ln)
        if m and out["total"] is None:
            out["total"] = float(m.group(1))
        m = re.match(r"\s*(\d+)\s+iterations", ln)
        if m and out["iterations"] is None:
            out["iterations"] = int(m.group(1))
        if "Energy" in ln and "Strength" in ln and not out["table"]:
            for row in lines[i + 2:]:
                t = row.split()
                if len(t) != 2:
                    break
                try:
                    out["table"].append([float(t[0]), float(t[1])])
                except ValueError:
                    break
    return out


def read_expect(path):
    """<H> table of an expectation-value run: state, E, J, T^2, <H>, norm."""
    rows = []
    lines = open(path).read().splitlines()
    for i, ln in enumerate(lines):
        if "STATE" in ln and "<H >" in ln:
            for row in lines[i + 1:]:
                t = row.split()
                if len(t) != 6 or not t[0].isdigit():
                    break
                rows.append({"n": int(t[0]), "E": float(t[1]), "J": float(t[2]), "T2": float(t[3]),
                             "H": float(t[4]), "norm": float(t[5])})
            break
    return rows


def read_overlap(path):
    """overlap.dat: initial state, then per final state E, J, T, <i|f>, |<i|f>|^2."""
    lines = open(path).read().splitlines()
    init = int(lines[0].split("=")[1])
    rows = []
    for row in lines[2:]:
        t = row.split()
        if len(t) != 6:
            continue
        rows.append({"n": int(t[0]), "E": float(t[1]), "J": float(t[2]), "T": float(t[3]),
                     "overlap": float(t[4]), "overlap2": float(t[5])})
    return {"initial": init, "finals": rows}


def read_dres_m(path):
    """The Mathematica-form density file of a density-from-wavefunction run:
    state energies (8 decimals) and every (initial, final, Jt) block with
    rows [a, b, rho_Tt=0, rho_Tt=1] (8 decimals)."""
    txt = open(path).read()
    states = re.search(r"densSetStates\[\{(.*?)\}\];", txt, re.S).group(1)
    energies = [float(r.split(",")[1]) for r in re.findall(r"\{([^{}]*)\}", states) if r.strip()[:1].isdigit()]
    blocks = []
    for m in re.finditer(r"densMatElem\[\s*(\d+),\s*(\d+),\s*(\d+),\s*\{(.*?)\}\];", txt, re.S):
        rows = [[float(x) for x in r.split(",")] for r in re.findall(r"\{([^{}]*)\}", m.group(4))]
        if rows:
            blocks.append({"i": int(m.group(1)), "f": int(m.group(2)), "Jt": int(m.group(3)),
                           "rho": [[int(r[0]), int(r[1]), r[2], r[3]] for r in rows]})
    return {"energies": energies, "blocks": blocks}


def read_input(path):
    toks = [ln.split("!")[0].split() for ln in open(path)]
    toks = [t for t in toks if t]
    # d / name / sps / "Z N" / 2Jz / n / int / scaling / end / ld / nkeep niter
    zn = [int(x) for x in toks[3][:2]]
    jz2 = int(toks[4][0])
    scaling = [float(x) for x in toks[7][:4]]
    nkeep, niter = (int(x) for x in toks[10][:2])
    return {"np": zn[0], "nn": zn[1], "jz2": jz2, "scaling": scaling, "nkeep": nkeep, "niter": niter}


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference checkout> (the BIGSTICK source tree holding examples/sd)")
    ref = sys.argv[1]
    ex = os.path.join(ref, "examples", "sd")
    orbits = model.read_sps(os.path.join(ex, "sd.sps"))
    spe, tbme = model.read_int(os.path.join(ex, "usdb.int"), len(orbits))
    out = {"source": "examples/sd of the BIGSTICK reference (sd.sps, usdb.int, input.mg25*, output/*.res)",
           "orbits": orbits, "spe": spe, "tbme": tbme, "runs": {}}
    for name, inp in (("mg25ref", "input.mg25ref"), ("mg25alt", "input.mg25altwfn")):
        states, iters = read_res(os.path.join(ex, "output", name + ".res"))
        run = read_input(os.path.join(ex, inp))
        run.update({"states": states, "reference_iterations": iters,
                    "res_file": f"examples/sd/output/{name}.res",
                    "density_jt0": read_diag_density(os.path.join(ex, "output", name + ".res")),
                    "densities": read_all_densities(os.path.join(ex, "output", name + ".res"))})
        out["runs"][name] = run
    out["expect_h"] = {"res_file": "examples/sd/output/mg25expectH.res",
                       "of": "the 10 mg25ref states under the mg25ref Hamiltonian (input.mg25expectH)",
                       "states": read_expect(os.path.join(ex, "output", "mg25expectH.res"))}
    out["overlap"] = dict(read_overlap(os.path.join(ex, "output", "overlap.dat")),
                          file="examples/sd/output/overlap.dat",
                          of="state 1 of mg25ref against the 10 mg25alt states (input.mg25overlap)")
    out["density_8dec"] = dict(read_dres_m(os.path.join(ex, "output", "mg25dx_dres.m")),
                               file="examples/sd/output/mg25dx_dres.m",
                               of="one-body densities of the 10 mg25ref states from their wavefunction file "
                                  "(input.mg25denfromwfn), 8 decimals")
    out["spin_operator"] = {"file": "examples/sd/sdspin.opme",
                            "text": open(os.path.join(ex, "sdspin.opme")).read()}
    st = read_strength(os.path.join(ex, "output", "mg25spinstrength1.res"))
    st.update({"res_file": "examples/sd/output/mg25spinstrength1.res",
               "pivot": "state 1 of mg25ref with the operator of sdspin.opme applied (input.mg25apply1b, "
                        "input.mg25strength)", "scaling": [1.0, 18.0, 25.0, 0.3]})
    out["spin_strength"] = st
    with open(os.path.join(HERE, "mg25.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", os.path.join(HERE, "mg25.json"))


if __name__ == "__main__":
    main()
